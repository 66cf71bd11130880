// Ragged columns with u64 offsets in the cs:: runtime (compiled by cospanmdao_b200.examples.build_runtime_tests, run by
// tests/test_examples_gpu.py). The reference's columns are u32 and reject a total past 2^32 - 1
// (cospanmdao/include/naga/cospan/shape_hook.hpp:455-457); its roadmap names the offset type as a parameter
// (internal/ROADMAP.md:106). Here:
//   - counts_from<std::uint64_t> builds a column whose total is 2^32 + 11 u8 elements (about 4.3 GB each for the
//     hooked layout and the output), and a component reads every block where the offsets put it: each block's first
//     and last element, its size, and its start relative to block 0 (a u32 offset would have wrapped block 2 onto
//     block 0);
//   - the default counts_from (u32 offsets) refuses the same counts with an error that names the u64 form;
//   - host counts (a producer's set_shape) past 2^32 - 1 take u64 offsets by themselves.
// Prints one line per case and "ALL OK" when every case passes; exits 1 otherwise.
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "naga/cospan/cospan.hpp"

namespace cs = naga::cospan;
using cs::DType;

namespace rw {

constexpr std::uint64_t kBig0 = (1ull << 31) + 3, kBig1 = (1ull << 31) + 1, kSmall = 7;  // total 2^32 + 11

int g_fails = 0;
void check(bool ok, const std::string& what) {
    if (!ok) {
        std::printf("  FAIL: %s\n", what.c_str());
        ++g_fails;
    }
}

// pts takes the hooked layout's shape; block i gets i + 1 in its first element and 101 + i in its last
class Mark : public cs::Component<Mark> {
public:
    struct Inputs {
        cs::Input<DType::u64, 1> cnt;
        cs::RaggedInput<DType::u8, 2> layout;
    };
    struct Outputs { cs::RaggedOutput<DType::u8, 2> pts; };
    __host__ __device__ static void compute_forward(sycl::id<1> id, const Inputs&, const Outputs& out) {
        auto b = out.pts.block(id[0]);
        if (b.size() == 0) return;
        b[0] = static_cast<std::uint8_t>(1 + id[0]);
        b[b.size() - 1] = static_cast<std::uint8_t>(101 + id[0]);
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.cnt, "cnt", 3);
        declare_input(inputs.layout, "layout");
        declare_output(outputs.pts, "pts");
    }
    void prepare_forward() override { set_shape(outputs.pts, shape_of(inputs.layout)); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(sycl::range<1>{inputs.layout.size()}));
    }
};

// the same output from host counts given in prepare_forward
class MarkHost : public cs::Component<MarkHost> {
public:
    struct Inputs {};
    struct Outputs { cs::RaggedOutput<DType::u8, 2> pts; };
    __host__ __device__ static void compute_forward(sycl::id<1> id, const Inputs&, const Outputs& out) {
        auto b = out.pts.block(id[0]);
        if (b.size() == 0) return;
        b[0] = static_cast<std::uint8_t>(1 + id[0]);
        b[b.size() - 1] = static_cast<std::uint8_t>(101 + id[0]);
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override { declare_output(outputs.pts, "pts"); }
    void prepare_forward() override { set_shape(outputs.pts, 3, std::vector<std::size_t>{kBig0, kBig1, kSmall}); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(sycl::range<1>{3}));
    }
};

// info[4 i ..]: block i's first element, last element, size, and start relative to block 0
class Probe : public cs::Component<Probe> {
public:
    struct Inputs { cs::RaggedInput<DType::u8, 2> pts; };
    struct Outputs { cs::Output<DType::u64, 1> info; };
    __host__ __device__ static void compute_forward(sycl::id<1> id, const Inputs& in, const Outputs& out) {
        const std::size_t i = id[0];
        auto b = in.pts.block(i);
        const std::size_t n = b.size();
        out.info[sycl::id<1>{4 * i + 0}] = n ? b[0] : 0;
        out.info[sycl::id<1>{4 * i + 1}] = n ? b[n - 1] : 0;
        out.info[sycl::id<1>{4 * i + 2}] = n;
        out.info[sycl::id<1>{4 * i + 3}] = static_cast<std::uint64_t>(b.data_ - in.pts.block(0).data_);
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.pts, "pts");
        declare_output(outputs.info, "info", cs::unspecified);
    }
    void prepare_forward() override { set_shape(outputs.info, 4 * shape_of(inputs.pts).n); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(sycl::range<1>{inputs.pts.size()}));
    }
};

template <bool Wide>
class HookTop : public cs::System {
public:
    void setup() override {
        add_subsystem(cs::subsystem_desc<Mark>("mark"));
        add_subsystem(cs::subsystem_desc<Probe>("probe"));
        connect("mark.pts", "probe.pts");
        if constexpr (Wide) shape_hook("mark.layout", cs::ragged::counts_from<std::uint64_t>("mark.cnt"));
        else shape_hook("mark.layout", cs::ragged::counts_from("mark.cnt"));
    }
};

class HostTop : public cs::System {
public:
    void setup() override {
        add_subsystem(cs::subsystem_desc<MarkHost>("mark"));
        add_subsystem(cs::subsystem_desc<Probe>("probe"));
        connect("mark.pts", "probe.pts");
    }
};

void expect_info(cs::Model& m, const std::string& name) {
    auto v = m.view_output<DType::u64, 1>("probe.info");
    v.sync();
    auto s = v.span();
    const std::vector<std::uint64_t> want = {1, 101, kBig0, 0,            2, 102, kBig1, kBig0,
                                             3, 103, kSmall, kBig0 + kBig1};
    check(s.size() == want.size(), name + ": 12 probe values");
    for (std::size_t k = 0; k < want.size() && k < s.size(); ++k)
        if (s[k] != want[k]) {
            std::printf("  FAIL: %s: info[%zu] = %llu, want %llu\n", name.c_str(), k, (unsigned long long)s[k],
                        (unsigned long long)want[k]);
            ++g_fails;
        }
}

void case_hook_u64() {
    cs::Model m = cs::create_model<HookTop<true>>();
    m.setup();
    m.update_input("mark.cnt", cs::init::from_host(std::vector<std::uint64_t>{kBig0, kBig1, kSmall}));
    m.run();
    m.wait();
    expect_info(m, "counts_from<u64>");
}

void case_hook_u32_refuses() {
    std::string msg;
    try {
        cs::Model m = cs::create_model<HookTop<false>>();
        m.setup();
        m.update_input("mark.cnt", cs::init::from_host(std::vector<std::uint64_t>{kBig0, kBig1, kSmall}));
        m.run();
        m.wait();
    } catch (const std::exception& e) {
        msg = e.what();
    }
    check(msg.find("2^32 - 1") != std::string::npos && msg.find("counts_from<std::uint64_t>") != std::string::npos,
          "u32 offsets refuse a total past 2^32 - 1 (got: " + msg + ")");
}

void case_host_counts() {
    cs::Model m = cs::create_model<HostTop>();
    m.setup();
    m.run();
    m.wait();
    expect_info(m, "host counts");
}

int run(const char* name, void (*f)()) {
    const int before = g_fails;
    try {
        f();
    } catch (const std::exception& e) {
        std::printf("  FAIL: exception: %s\n", e.what());
        ++g_fails;
    }
    std::printf("%-40s %s\n", name, g_fails == before ? "OK" : "FAIL");
    return g_fails == before ? 0 : 1;
}

}  // namespace rw

int main() {
    int fails = 0;
    fails += rw::run("counts_from<u64>, total 2^32 + 11", rw::case_hook_u64);
    fails += rw::run("counts_from (u32) refuses it", rw::case_hook_u32_refuses);
    fails += rw::run("host counts widen by themselves", rw::case_host_counts);
    std::printf(fails ? "FAILED\n" : "ALL OK\n");
    return fails ? 1 : 0;
}
