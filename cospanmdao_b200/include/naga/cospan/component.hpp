// naga/cospan/component.hpp — cs::Component<X> and the kernels that run component bodies on the GPU.
//
// A component declares ports in declare(), sizes its outputs in prepare_forward(), and says how it launches in
// define_forward() (reference: component.hpp:178-749, :1106-1132, :1438-1485). Its static compute_forward is the body:
// its first parameter fixes the kind — sycl::id<R> (one work-item per index) or cs::GroupItem<R> (work-groups, with an
// optional cs::LocalMem as the fourth parameter).
//
// On this backend a bare component is one CUDA launch (grid-stride over its indices or its work-groups), and a fused
// group of group-range stages is one cooperative launch that runs its segments in order: within a segment every
// work-group runs the segment's stages one after the other (in local memory they share or partition), and a grid
// barrier — bounded, like every wait here — separates segments. That order is at least as strong as the reference's
// tickets (kernel.hpp:215-236), so wait_group() has nothing left to wait for.
#pragma once

#include <cxxabi.h>

#include <cstdlib>
#include <map>
#include <string>
#include <typeinfo>

#include "core.hpp"

namespace naga::cospan {

class Model;
class System;
namespace detail {
class Runtime;
struct Var;
}  // namespace detail

// ---- the tree -----------------------------------------------------------------------------------------------------
class Node {
public:
    enum class Kind { system, component, fused };
    virtual ~Node() = default;
    std::string name;
    Node* parent = nullptr;
    Kind kind = Kind::system;
    std::string path() const {
        if (!parent) return name;
        const std::string p = parent->path();
        return p.empty() ? name : p + "." + name;
    }
};

namespace detail {
inline std::string demangle(const char* n) {
    int st = 0;
    char* d = abi::__cxa_demangle(n, nullptr, nullptr, &st);
    std::string r = (st == 0 && d) ? d : n;
    std::free(d);
    return r;
}

// one port of a component: its name, dtype, rank, declared shape, and how to point its wrapper at a variable
struct PortRec {
    std::string name;
    bool output = false;
    DType dtype = DType::f32;
    int rank = 1;
    ShapeSpec declared;
    std::function<void(void*, const std::size_t*)> bind;
    const void* wrapper = nullptr;
    int var = -1;
    // a ragged port: declared counts (cs::counts / cs::offsets) and how to point its wrapper at a variable (data, N,
    // block offsets and per-index extents on the device, or nullptr and the row length for a dense variable)
    bool ragged = false;
    std::optional<std::vector<std::size_t>> counts;
    std::function<void(void*, std::size_t, const std::uint32_t*, const std::uint64_t*, const std::uint32_t*, std::size_t)>
        bind_ragged;
};

inline std::string list_of(const std::vector<std::size_t>& v) {
    std::string s = "[";
    for (std::size_t i = 0; i < v.size(); ++i) s += (i ? "," : "") + std::to_string(v[i]);
    return s + "]";
}

template <class S>
inline void spec_from(ShapeSpec& s, int& d, const S& v) {
    if constexpr (std::is_same_v<S, Unspecified>) {
        s.known[d++] = false;
    } else if constexpr (std::is_integral_v<S>) {
        s.ext[d] = static_cast<std::size_t>(v);
        s.known[d++] = true;
    } else {  // std::array<Unspecified, R>
        for (std::size_t k = 0; k < std::tuple_size_v<S>; ++k) s.known[d++] = false;
    }
}
template <int R, class... S>
ShapeSpec declared_shape(const S&... s) {
    ShapeSpec sp;
    sp.rank = R;
    if constexpr (sizeof...(S) > 0) {
        int d = 0;
        (spec_from(sp, d, s), ...);
        if (d != R) throw std::invalid_argument("naga::cospan: declared shape has the wrong number of dimensions");
    }
    return sp;
}

// ---- body traits ----
template <class F> struct body_traits;
template <class It, class In, class Out>
struct body_traits<void (*)(It, const In&, const Out&)> {
    using item = It;
    using local = void;
};
template <class It, class In, class Out, class LM>
struct body_traits<void (*)(It, const In&, const Out&, LM)> {
    using item = It;
    using local = LM;
};
template <class T> struct item_kind;
template <int R> struct item_kind<sycl::id<R>> {
    static constexpr bool group = false;
    static constexpr int rank = R;
};
template <int R> struct item_kind<GroupItem<R>> {
    static constexpr bool group = true;
    static constexpr int rank = R;
};
template <class X> using body_t = body_traits<decltype(&X::compute_forward)>;
template <class X> inline constexpr bool is_group_body = item_kind<typename body_t<X>::item>::group;
template <class X> inline constexpr int body_rank = item_kind<typename body_t<X>::item>::rank;
template <class X> using body_local_t = typename body_t<X>::local;

// where a stage's local arrays start in the launch's dynamic shared memory
struct LocalLayout {
    std::uint32_t base = 0;  // bytes into the dynamic shared memory
    std::array<std::array<std::size_t, 3>, 8> shapes{};
    std::array<std::size_t, 8> offsets{};
};

template <class LM>
__device__ inline LM make_local(unsigned char* smem, const LocalLayout& L) {
    LM lm;
    lm.base = smem + L.base;
    for (std::size_t i = 0; i < lm.shapes.size(); ++i) {
        lm.shapes[i] = L.shapes[i];
        lm.offsets[i] = L.offsets[i];
    }
    return lm;
}

template <int R>
__device__ inline sycl::id<R> delinear(std::uint64_t l, const sycl::range<R>& r) {
    sycl::id<R> g;
    for (int d = R - 1; d >= 0; --d) {
        g[d] = l % r[d];
        l /= r[d];
    }
    return g;
}

// ---- bare launches ----
template <class X, int R>
__global__ void k_index(typename X::Inputs in, typename X::Outputs out, sycl::range<R> r, std::uint64_t total) {
    for (std::uint64_t t = std::uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += std::uint64_t(gridDim.x) * blockDim.x)
        X::compute_forward(delinear<R>(t, r), in, out);
}

template <class X, int R>
__global__ void k_group(typename X::Inputs in, typename X::Outputs out, sycl::range<R> groups, sycl::range<R> local,
                        std::uint64_t count, LocalLayout L) {
    extern __shared__ __align__(16) unsigned char cs_smem[];
    for (std::uint64_t g = blockIdx.x; g < count; g += gridDim.x) {
        GroupItem<R> it;
        it.group_id = delinear<R>(g, groups);
        it.group_range = groups;
        it.local_range = local;
        if constexpr (std::is_void_v<body_local_t<X>>) X::compute_forward(it, in, out);
        else X::compute_forward(it, in, out, make_local<body_local_t<X>>(cs_smem, L));
        __syncthreads();
    }
}
}  // namespace detail

// ---- components ---------------------------------------------------------------------------------------------------
class ComponentBase : public Node {
public:
    ComponentBase() { kind = Kind::component; }
    virtual void declare() {}
    virtual void prepare_forward() {}
    virtual std::unique_ptr<LaunchDescription> define_forward() { return nullptr; }

    // ---- runtime side ----
    std::vector<detail::PortRec> ports_;
    std::vector<std::pair<std::string, InitSpec>> own_inits_;
    std::string type_name_;
    detail::Runtime* rt_ = nullptr;
    virtual bool group_body() const = 0;
    virtual int body_rank() const = 0;
    virtual std::vector<std::size_t> local_elem_sizes() const = 0;
    virtual void launch_solo(detail::Runtime& rt, const LaunchDescription& d) = 0;
    detail::PortRec* port(const std::string& n) {
        for (auto& p : ports_)
            if (p.name == n) return &p;
        return nullptr;
    }
    std::string describe() const { return path(); }

protected:
    template <DType DT, int R, class... S>
    void declare_input(Input<DT, R>& w, std::string name, const S&... shape) {
        add_port(std::move(name), false, DT, R, detail::declared_shape<R>(shape...), [&w](void* d, const std::size_t* s) {
            w.data_ = static_cast<const cpp_type_t<DT>*>(d);
            set_dims<R>(w.shape_, w.stride_, s);
        }, &w);
    }
    template <DType DT, int R, class... S>
    void declare_output(Output<DT, R>& w, std::string name, const S&... shape) {
        add_port(std::move(name), true, DT, R, detail::declared_shape<R>(shape...), [&w](void* d, const std::size_t* s) {
            w.data_ = static_cast<cpp_type_t<DT>*>(d);
            set_dims<R>(w.shape_, w.stride_, s);
        }, &w);
    }
    // ragged ports (component.hpp:220-260 of the reference): (m, name) both dimensions unspecified; (m, name, n) N
    // given; (m, name, cs::counts(v)) host counts, which give N too; (m, name, cs::offsets(v)) the same as offsets
    template <DType DT, int R>
    void declare_input(RaggedInput<DT, R>& w, std::string name) { add_ragged_port(w, std::move(name), false, {}, {}); }
    template <DType DT, int R, class N, std::enable_if_t<std::is_integral_v<N>, int> = 0>
    void declare_input(RaggedInput<DT, R>& w, std::string name, N n) {
        add_ragged_port(w, std::move(name), false, leading(n), {});
    }
    template <DType DT, int R>
    void declare_input(RaggedInput<DT, R>& w, std::string name, Counts c) {
        add_ragged_port(w, std::move(name), false, {}, std::move(c.v));
    }
    template <DType DT, int R>
    void declare_input(RaggedInput<DT, R>& w, std::string name, const Offsets& o) {
        add_ragged_port(w, std::move(name), false, {}, counts_of(o).v);
    }
    template <DType DT, int R>
    void declare_output(RaggedOutput<DT, R>& w, std::string name) { add_ragged_port(w, std::move(name), true, {}, {}); }
    template <DType DT, int R, class N, std::enable_if_t<std::is_integral_v<N>, int> = 0>
    void declare_output(RaggedOutput<DT, R>& w, std::string name, N n) {
        add_ragged_port(w, std::move(name), true, leading(n), {});
    }
    template <DType DT, int R>
    void declare_output(RaggedOutput<DT, R>& w, std::string name, Counts c) {
        add_ragged_port(w, std::move(name), true, {}, std::move(c.v));
    }
    template <DType DT, int R>
    void declare_output(RaggedOutput<DT, R>& w, std::string name, const Offsets& o) {
        add_ragged_port(w, std::move(name), true, {}, counts_of(o).v);
    }
    void init_input(std::string name, InitSpec init) { own_inits_.emplace_back(std::move(name), std::move(init)); }
    template <DType DT, int R>
    sycl::range<R> shape_of(const Input<DT, R>& w) const;
    template <DType DT, int R, class... E>
    void set_shape(Output<DT, R>& w, E... e);
    // a ragged port's shape: N, the total and the counts (on the device for a hooked or copied column)
    template <DType DT, int R>
    RaggedShape shape_of(const RaggedInput<DT, R>& w) const { return ragged_shape_of(&w); }
    template <DType DT, int R>
    RaggedShape shape_of(const RaggedOutput<DT, R>& w) const { return ragged_shape_of(&w); }
    /// A ragged output takes a RaggedShape (another port's, read with shape_of): N and the counts, device ones shared.
    template <DType DT, int R>
    void set_shape(RaggedOutput<DT, R>& w, const RaggedShape& s) { set_ragged_shape(&w, s); }
    /// A ragged output takes N and host counts (counts.size() == n).
    template <DType DT, int R, class N, std::enable_if_t<std::is_integral_v<N>, int> = 0>
    void set_shape(RaggedOutput<DT, R>& w, N n, std::vector<std::size_t> counts) {
        if (std::size_t(leading(n)) != counts.size())
            throw std::invalid_argument("naga::cospan: set_shape on '" + path() + "': N is " + std::to_string(n) + " but " +
                                        std::to_string(counts.size()) + " counts were given");
        RaggedShape s;
        s.n = counts.size();
        for (auto c : counts) s.total += c;
        s.counts = std::move(counts);
        set_ragged_shape(&w, s);
    }
    template <class... D>
    std::unique_ptr<LaunchDescription> create_launch_config(const D&... descs) const {
        auto L = std::make_unique<LaunchDescription>();
        (apply(*L, descs), ...);
        return L;
    }

private:
    RaggedShape ragged_shape_of(const void* wrapper) const;               // model.hpp
    void set_ragged_shape(const void* wrapper, const RaggedShape& s);     // model.hpp
    template <class N>
    static std::size_t leading(N n) {
        if constexpr (std::is_signed_v<N>)
            if (n < 0) throw std::invalid_argument("naga::cospan: a ragged port's N cannot be negative");
        return static_cast<std::size_t>(n);
    }
    template <class W>
    void add_ragged_port(W& w, std::string name, bool out, std::optional<std::size_t> n,
                         std::optional<std::vector<std::size_t>> counts) {
        ShapeSpec sp;
        sp.rank = 2;
        if (counts) n = counts->size();
        if (n) {
            sp.ext[0] = *n;
            sp.known[0] = true;
        }
        add_port(std::move(name), out, W::dtype, 2, sp, nullptr, &w);
        detail::PortRec& p = ports_.back();
        p.ragged = true;
        p.counts = std::move(counts);
        p.bind_ragged = [&w](void* d, std::size_t nb, const std::uint32_t* offs, const std::uint64_t* offs64,
                             const std::uint32_t* ext, std::size_t row) {
            w.data_ = static_cast<std::remove_reference_t<decltype(*w.data_)>*>(d);
            w.n_ = nb;
            w.offs_ = offs;
            w.offs64_ = offs64;
            w.ext_ = ext;
            w.row_ = row;
        };
    }
    template <int R>
    static void set_dims(sycl::range<R>& shape, sycl::range<R>& stride, const std::size_t* s) {
        std::size_t st = 1;
        for (int d = R - 1; d >= 0; --d) {
            shape[d] = s[d];
            stride[d] = st;
            st *= s[d];
        }
    }
    void add_port(std::string name, bool out, DType dt, int rank, ShapeSpec sp,
                  std::function<void(void*, const std::size_t*)> bind, const void* wrapper) {
        if (port(name))
            throw std::invalid_argument("naga::cospan: '" + path() + "' declares the port '" + name + "' twice");
        detail::PortRec p;
        p.name = std::move(name);
        p.output = out;
        p.dtype = dt;
        p.rank = rank;
        p.declared = sp;
        p.bind = std::move(bind);
        p.wrapper = wrapper;
        ports_.push_back(std::move(p));
    }
    template <int R>
    static void apply(LaunchDescription& L, const RangeDesc<R>& d) {
        L.rank = R;
        for (int k = 0; k < R; ++k) L.range[k] = d.r[k];
    }
    template <int R>
    static void apply(LaunchDescription& L, const WgDesc<R>& d) {
        L.has_wg = true;
        for (int k = 0; k < R; ++k) L.wg[k] = d.r[k];
    }
    static void apply(LaunchDescription& L, const LocalDesc& d) {
        L.local = d.shapes;
        L.local_ranks = d.ranks;
    }
};

template <class X>
class Component : public ComponentBase {
public:
    Component() { type_name_ = detail::demangle(typeid(X).name()); }
    bool group_body() const override { return detail::is_group_body<X>; }
    int body_rank() const override { return detail::body_rank<X>; }
    std::vector<std::size_t> local_elem_sizes() const override {
        using LM = detail::body_local_t<X>;
        if constexpr (std::is_void_v<LM>) return {};
        else {
            auto a = detail::local_arrays<LM>::elem_sizes();
            return std::vector<std::size_t>(a.begin(), a.end());
        }
    }
    void launch_solo(detail::Runtime& rt, const LaunchDescription& d) override;
};

// ---- fused-group descriptors (fused_component.hpp:460-569) ----------------------------------------------------------
struct group_waits_enabled {};
namespace range_split {
struct flatten_and_split {};
struct pad_and_split {};
struct padded {};
}  // namespace range_split
namespace local_mem {
struct partitioned {};
struct shared {};
}  // namespace local_mem
namespace range_mode {
struct own {};
struct whole {};
}  // namespace range_mode

template <class T, class... Args>
struct SubsystemDesc {
    std::string name;
    std::tuple<std::decay_t<Args>...> args;
    std::unique_ptr<T> make() const {
        return std::apply([](const auto&... a) { return std::make_unique<T>(a...); }, args);
    }
};
template <class T, class... Args>
SubsystemDesc<T, Args...> subsystem_desc(std::string name, Args&&... args) {
    return SubsystemDesc<T, Args...>{std::move(name), std::tuple<std::decay_t<Args>...>(std::forward<Args>(args)...)};
}

template <class Opts, class... Descs>
struct SegmentDesc {
    std::tuple<Descs...> descs;
};
template <class... Opts, class... Descs>
auto segment(Descs... d) {
    return SegmentDesc<std::tuple<Opts...>, Descs...>{std::tuple<Descs...>(std::move(d)...)};
}
struct GlobalBarrierDesc {};
inline GlobalBarrierDesc global_barrier() { return {}; }

struct ConnectsDesc {
    std::vector<std::pair<std::string, std::string>> pairs;
};
inline ConnectsDesc connects_desc(std::initializer_list<std::pair<std::string_view, std::string_view>> pairs) {
    ConnectsDesc c;
    for (auto& [a, b] : pairs) c.pairs.emplace_back(std::string(a), std::string(b));
    return c;
}
enum class TieOutputsPolicy : std::uint8_t { require_atomic, allow_plain };
struct TieEntry {
    std::vector<std::string> members;
    std::string name;
    ShapeSpec shape;
    bool outputs = false;
    TieOutputsPolicy policy = TieOutputsPolicy::require_atomic;
    DType dtype = DType::f32;
    int rank = 1;
};
struct TiesDesc {
    std::vector<TieEntry> entries;
};
inline TiesDesc ties_desc(std::initializer_list<TieEntry> entries) { return TiesDesc{std::vector<TieEntry>{entries}}; }
template <DType DT, int R>
TieEntry tie_inputs(std::initializer_list<std::string_view> members, std::string name, ShapeSpec shape = {}) {
    TieEntry t;
    for (auto m : members) t.members.emplace_back(m);
    t.name = std::move(name);
    t.shape = shape;
    t.dtype = DT;
    t.rank = R;
    return t;
}
template <DType DT, int R>
TieEntry tie_outputs(std::initializer_list<std::string_view> members, std::string name, ShapeSpec shape = {},
                     TieOutputsPolicy policy = TieOutputsPolicy::require_atomic) {
    TieEntry t = tie_inputs<DT, R>(members, std::move(name), shape);
    t.outputs = true;
    t.policy = policy;
    return t;
}

}  // namespace naga::cospan
