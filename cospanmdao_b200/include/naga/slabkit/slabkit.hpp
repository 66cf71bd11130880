// naga/slabkit/slabkit.hpp — the part of SlabKit's queue API that CoSpan initializers use
// (sk::unordered_queue::parallel_for(dev, deps, range, f), single_task), on the runtime's CUDA stream.
#pragma once

#include <vector>

#include <sycl/sycl.hpp>

namespace naga::slabkit {

class unordered_queue {
public:
    explicit unordered_queue(cudaStream_t s = nullptr) : s_(s) {}
    template <int D, class F>
    sycl::event parallel_for(const sycl::device&, const std::vector<sycl::event>& deps, sycl::range<D> r, F f) {
        sycl::handler h(s_);
        h.depends_on(deps);
        h.parallel_for(r, f);
        return sycl::event(s_);
    }
    template <class F>
    sycl::event single_task(const sycl::device&, const std::vector<sycl::event>& deps, F f) {
        sycl::handler h(s_);
        h.depends_on(deps);
        h.single_task(f);
        return sycl::event(s_);
    }
    cudaStream_t native() const { return s_; }

private:
    cudaStream_t s_;
};

}  // namespace naga::slabkit
