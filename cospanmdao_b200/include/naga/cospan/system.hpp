// naga/cospan/system.hpp — cs::System (a node that groups and wires children) and fused groups.
//
// The wiring calls record what the reference's System records (system.hpp:99-646, wiring.hpp:287-540): connect
// (a consumer reads a producer's variable), promote (a name in this system for a descendant's port), tie_inputs /
// tie_outputs (several ports share one variable, with a shape), shape_hook, init_input. Names resolve when the model
// finalizes (model.hpp). fuse_components builds a FusedGroup<Items...>: a leaf that owns its stages and runs them
// in one launch (fused_component.hpp:372-569).
#pragma once

#include <map>
#include <string_view>
#include <variant>

#include "component.hpp"

namespace naga::cospan {

class ShapeHookCtx;  // what a custom descriptor reads through (model.hpp)

// shape-hook descriptors (shape_hook.hpp:65-84): one per dimension, or one ragged descriptor for a rank-2 target
namespace dim {
struct AsIs {};
struct FixedAtRun { std::size_t v = 0; };
struct FromShape { std::string path; std::size_t d = 0; };
struct FromValue { std::string path; std::size_t index = 0; };
struct Custom { std::function<std::size_t(ShapeHookCtx&)> fn; };
inline AsIs as_is() { return {}; }
inline FixedAtRun fixed_at_run(std::size_t v) { return FixedAtRun{v}; }
inline FromShape from_shape(std::string path, std::size_t d) { return FromShape{std::move(path), d}; }
/// the VALUE of element `index` (flat) of an integer variable
inline FromValue from_value(std::string path, std::size_t index) { return FromValue{std::move(path), index}; }
inline Custom custom(std::function<std::size_t(ShapeHookCtx&)> fn) { return Custom{std::move(fn)}; }
}  // namespace dim
namespace ragged {
/// the per-index counts are the values of an integer variable (rank 1 [N], or column 0 of a rank-2 [N, k])
struct CountsFrom { std::string path; bool wide = false; };
/// the N + 1 block offsets are the values of a rank-1 integer variable
struct OffsetsFrom { std::string path; bool wide = false; };
/// Offset is the column's offset type: std::uint32_t (the reference's, and the default: the total stays below 2^32)
/// or std::uint64_t (a total past 2^32 - 1, at 8 bytes per offset). Extents are u32 either way.
template <class Offset = std::uint32_t>
inline CountsFrom counts_from(std::string path) {
    static_assert(std::is_same_v<Offset, std::uint32_t> || std::is_same_v<Offset, std::uint64_t>,
                  "naga::cospan: a ragged column's offsets are std::uint32_t or std::uint64_t");
    return CountsFrom{std::move(path), sizeof(Offset) == 8};
}
template <class Offset = std::uint32_t>
inline OffsetsFrom offsets_from(std::string path) {
    static_assert(std::is_same_v<Offset, std::uint32_t> || std::is_same_v<Offset, std::uint64_t>,
                  "naga::cospan: a ragged column's offsets are std::uint32_t or std::uint64_t");
    return OffsetsFrom{std::move(path), sizeof(Offset) == 8};
}
}  // namespace ragged
using HookDim = std::variant<dim::AsIs, dim::FixedAtRun, dim::FromShape, dim::FromValue, dim::Custom, ragged::CountsFrom,
                             ragged::OffsetsFrom>;

class System : public Node {
public:
    System() { kind = Kind::system; }
    virtual void setup() {}

    template <class T, class... A>
    void add_subsystem(const SubsystemDesc<T, A...>& d) {
        std::unique_ptr<T> c = d.make();
        adopt(std::move(c), d.name);
    }
    template <class D, class = decltype(std::declval<const D&>().build())>
    void add_subsystem(const D& d) {
        adopt(d.build(), d.name);
    }

    /// Records a connect. The ragged wiring rules are checked in the call, as the reference does (wiring.hpp): a dense
    /// Input cannot read a ragged source, and two ragged ports that both declare N or counts must agree.
    void connect(std::string_view src, std::string_view dst) {
        check_ragged_connect(std::string(src), std::string(dst));
        connects_.emplace_back(std::string(src), std::string(dst));
    }
    template <DType DT, int R>
    void promote(std::string_view path, std::string alias) {
        if (aliases_.count(alias))
            throw std::invalid_argument("naga::cospan: '" + this->path() + "' promotes the name '" + alias + "' twice");
        aliases_[alias] = Alias{std::string(path), DT, R};
    }
    template <DType DT, int R>
    void tie_inputs(std::initializer_list<std::string_view> members, std::string name, ShapeSpec shape = {}) {
        ties_.push_back(cs_tie_inputs<DT, R>(members, std::move(name), shape));
    }
    template <DType DT, int R>
    void tie_outputs(std::initializer_list<std::string_view> members, std::string name, ShapeSpec shape = {},
                     TieOutputsPolicy policy = TieOutputsPolicy::require_atomic) {
        TieEntry t = cs_tie_inputs<DT, R>(members, std::move(name), shape);
        t.outputs = true;
        t.policy = policy;
        ties_.push_back(std::move(t));
    }
    template <class... D>
    void shape_hook(std::string_view path, D... dims) {
        hooks_.push_back(Hook{std::string(path), std::vector<HookDim>{HookDim(std::move(dims))...}});
    }
    void init_input(std::string_view path, InitSpec init) { inits_.emplace_back(std::string(path), std::move(init)); }

    Node* child(const std::string& n) const {
        for (auto& c : children_)
            if (c->name == n) return c.get();
        return nullptr;
    }

    // ---- recorded structure (read by the model) ----
    struct Alias {
        std::string target;
        DType dtype;
        int rank;
    };
    struct Hook {
        std::string path;
        std::vector<HookDim> dims;
    };
    std::vector<std::unique_ptr<Node>> children_;
    std::vector<std::pair<std::string, std::string>> connects_;
    std::map<std::string, Alias> aliases_;
    std::vector<TieEntry> ties_;
    std::vector<Hook> hooks_;
    std::vector<std::pair<std::string, InitSpec>> inits_;

    void adopt(std::unique_ptr<Node> c, const std::string& name) {
        if (name.empty() || name.find('.') != std::string::npos)
            throw std::invalid_argument("naga::cospan: '" + path() + "': a child name must be non-empty and have no '.'");
        if (child(name)) throw std::invalid_argument("naga::cospan: '" + path() + "' already has a child '" + name + "'");
        c->name = name;
        c->parent = this;
        Node* raw = c.get();
        children_.push_back(std::move(c));
        if (raw->kind == Kind::component) static_cast<ComponentBase*>(raw)->declare();
        else static_cast<System*>(raw)->setup();
    }

    /// The port a path names below this system, through child names (nullptr when it names none of them).
    detail::PortRec* find_port(const std::string& path) const {
        const auto dot = path.find('.');
        if (dot == std::string::npos) return nullptr;
        Node* c = child(path.substr(0, dot));
        if (!c) return nullptr;
        const std::string rest = path.substr(dot + 1);
        if (c->kind == Kind::component) return static_cast<ComponentBase*>(c)->port(rest);
        return static_cast<System*>(c)->find_port(rest);
    }

private:
    void check_ragged_connect(const std::string& a, const std::string& b) const {
        const detail::PortRec* pa = find_port(a);
        const detail::PortRec* pb = find_port(b);
        if (!pa || !pb) return;  // promoted or tied names: checked when the model finalizes
        const std::string call = "naga::cospan: connect('" + a + "', '" + b + "')";
        auto dense_reader = [&](const detail::PortRec* src, const std::string& sn, const detail::PortRec* dst,
                                const std::string& dn) {
            if (src->ragged && src->output && !dst->ragged && !dst->output)
                throw std::invalid_argument(call + ": '" + sn + "' is ragged; a dense Input cannot see per-index extents "
                                            "(declare '" + dn + "' as a RaggedInput)");
        };
        dense_reader(pa, a, pb, b);
        dense_reader(pb, b, pa, a);
        if (!pa->ragged || !pb->ragged) return;
        if (pa->declared.known[0] && pb->declared.known[0] && pa->declared.ext[0] != pb->declared.ext[0])
            throw std::invalid_argument(call + ": dimension 0: '" + a + "' declares " + std::to_string(pa->declared.ext[0]) +
                                        ", '" + b + "' declares " + std::to_string(pb->declared.ext[0]) +
                                        "; the extents must match");
        if (pa->counts && pb->counts && *pa->counts != *pb->counts)
            throw std::invalid_argument(call + ": dimension 1: the counts must match ('" + a + "' declares " +
                                        detail::list_of(*pa->counts) + ", '" + b + "' declares " +
                                        detail::list_of(*pb->counts) + ")");
    }
    template <DType DT, int R>
    static TieEntry cs_tie_inputs(std::initializer_list<std::string_view> members, std::string name, ShapeSpec shape) {
        return naga::cospan::tie_inputs<DT, R>(members, std::move(name), shape);
    }
};

// system_from(name, items...): an ordinary System of the given children (fused_component.hpp:572-580)
template <class... Descs>
struct SystemFromDesc {
    std::string name;
    ConnectsDesc connects;
    std::tuple<Descs...> descs;
    std::unique_ptr<Node> build() const {
        auto s = std::make_unique<FromSystem>(connects, descs);
        return s;
    }
    struct FromSystem : System {
        ConnectsDesc c;
        std::tuple<Descs...> d;
        FromSystem(ConnectsDesc cc, std::tuple<Descs...> dd) : c(std::move(cc)), d(std::move(dd)) {}
        void setup() override {
            std::apply([this](const auto&... x) { (add_subsystem(x), ...); }, d);
            for (auto& [a, b] : c.pairs) connect(a, b);
        }
    };
};
template <class... Descs>
SystemFromDesc<Descs...> system_from(std::string name, ConnectsDesc c, Descs... d) {
    return SystemFromDesc<Descs...>{std::move(name), std::move(c), std::tuple<Descs...>(std::move(d)...)};
}
template <class... Descs>
SystemFromDesc<Descs...> system_from(std::string name, Descs... d) {
    return SystemFromDesc<Descs...>{std::move(name), ConnectsDesc{}, std::tuple<Descs...>(std::move(d)...)};
}

// ---- fused groups -----------------------------------------------------------------------------------------------
namespace detail {
template <class... T> struct tlist {};
template <class A, class B> struct tcat;
template <class... A, class... B> struct tcat<tlist<A...>, tlist<B...>> { using type = tlist<A..., B...>; };

// the component types of a fuse_components item list, flattened in order
template <class D> struct stages_of { using type = tlist<>; };
template <class T, class... A> struct stages_of<SubsystemDesc<T, A...>> { using type = tlist<T>; };
template <class O> struct stages_of<SegmentDesc<O>> { using type = tlist<>; };
template <class O, class D, class... Ds> struct stages_of<SegmentDesc<O, D, Ds...>> {
    using type = typename tcat<typename stages_of<D>::type, typename stages_of<SegmentDesc<O, Ds...>>::type>::type;
};
template <class... Ds> struct stages_of_all { using type = tlist<>; };
template <class D, class... Ds> struct stages_of_all<D, Ds...> {
    using type = typename tcat<typename stages_of<D>::type, typename stages_of_all<Ds...>::type>::type;
};

template <class T, class Tuple> struct has_opt;
template <class T, class... O> struct has_opt<T, std::tuple<O...>> : std::bool_constant<(std::is_same_v<T, O> || ...)> {};

constexpr int kMaxStages = 24;
constexpr int kMaxSegments = 16;

struct StageGeom {
    std::uint32_t segment = 0;
    std::uint32_t whole = 0;  // range_mode::whole
    std::uint64_t count = 0;  // the stage's own work-groups
    std::uint64_t items = 0;  // an index-range stage: its indices (groups holds its range)
    std::array<std::size_t, 3> groups{1, 1, 1};
    std::array<std::size_t, 3> local{1, 1, 1};
    LocalLayout local_mem;
};
struct SegGeom {
    std::uint64_t count = 0;  // work-groups of the segment's block (max over its stages)
};

template <class... Xs>
struct FusedParams {
    std::tuple<std::pair<typename Xs::Inputs, typename Xs::Outputs>...> io;
    StageGeom st[sizeof...(Xs)];
    SegGeom seg[kMaxSegments];
    std::uint32_t nseg = 0;
    std::uint32_t* ctrl = nullptr;  // barrier counters and status word
};

// bounded grid barrier (the same protocol as the cspb kernels: a status word records a timeout)
__device__ inline bool fused_barrier(std::uint32_t* ctrl) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        std::uint32_t* count = ctrl + 1;
        std::uint32_t* gen = ctrl + 2;
        const std::uint32_t g = *reinterpret_cast<volatile std::uint32_t*>(gen);
        __threadfence();
        const std::uint32_t arrived = atomicAdd(count, 1u);
        bool ok = true;
        if (arrived == gridDim.x - 1) {
            atomicExch(count, 0u);
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            unsigned long long t0, t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
            while (*reinterpret_cast<volatile std::uint32_t*>(gen) == g) {
                if (*reinterpret_cast<volatile std::uint32_t*>(ctrl) != 0u) { ok = false; break; }
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                if (t - t0 > 2000000000ull) {
                    atomicOr(ctrl, 1u);
                    ok = false;
                    break;
                }
                __nanosleep(64);
            }
            __threadfence();
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <class X, int I, class P>
__device__ inline void run_stage(const P& p, std::uint64_t lg, unsigned char* smem) {
    const StageGeom& g = p.st[I];
    if constexpr (!is_group_body<X>) {
        // an index-range stage: group lg of the segment runs indices [lg * threads, (lg + 1) * threads) of its
        // flattened range, one per work-item
        constexpr int R = body_rank<X>;
        const std::uint64_t t = lg * blockDim.x + threadIdx.x;
        if (lg >= g.count || t >= g.items) return;
        sycl::range<R> r;
        for (int d = 0; d < R; ++d) r[d] = g.groups[d];
        const auto& io = std::get<I>(p.io);
        X::compute_forward(delinear<R>(t, r), io.first, io.second);
        return;
    } else {
        // own: the stage runs for its first `count` groups of the segment's block; whole: for every group of the block
        const std::uint64_t cnt = g.whole ? p.seg[g.segment].count : g.count;
        if (lg >= cnt) return;
        constexpr int R = body_rank<X>;
        GroupItem<R> it;
        std::uint64_t rest = 1;
        for (int d = 0; d < R; ++d) {
            it.group_range[d] = g.groups[d];
            it.local_range[d] = g.local[d];
            if (d > 0) rest *= g.groups[d];
        }
        if (g.whole) it.group_range[0] = (cnt + rest - 1) / rest;
        it.group_id = delinear<R>(lg, it.group_range);
        it.segment = g.segment;
        const auto& io = std::get<I>(p.io);
        if constexpr (std::is_void_v<body_local_t<X>>) X::compute_forward(it, io.first, io.second);
        else X::compute_forward(it, io.first, io.second, make_local<body_local_t<X>>(smem, g.local_mem));
    }
}

template <class P, class... Xs, std::size_t... I>
__device__ inline void run_segment_stages(const P& p, std::uint32_t s, std::uint64_t lg, unsigned char* smem,
                                          std::index_sequence<I...>) {
    ((p.st[I].segment == s ? run_stage<Xs, int(I)>(p, lg, smem) : void()), ...);
}

template <class... Xs>
__global__ void k_fused(FusedParams<Xs...> p) {
    extern __shared__ __align__(16) unsigned char cs_smem[];
    for (std::uint32_t s = 0; s < p.nseg; ++s) {
        for (std::uint64_t lg = blockIdx.x; lg < p.seg[s].count; lg += gridDim.x) {
            run_segment_stages<FusedParams<Xs...>, Xs...>(p, s, lg, cs_smem, std::index_sequence_for<Xs...>{});
            __syncthreads();
        }
        if (s + 1 < p.nseg && !fused_barrier(p.ctrl)) return;
    }
}
}  // namespace detail

class FusedGroupBase : public System {
public:
    FusedGroupBase() { kind = Kind::fused; }
    std::vector<ComponentBase*> stages_;
    std::vector<int> stage_segment_;
    std::vector<int> segment_local_shared_;  // per segment: 1 local_mem::shared, 0 partitioned
    std::vector<int> segment_whole_;         // per segment: 1 range_mode::whole
    std::vector<int> segment_barrier_;       // per segment: a global_barrier stands before it
    virtual void launch(detail::Runtime& rt) = 0;
};

template <class Opts, class... Items>
class FusedGroup : public FusedGroupBase {
public:
    FusedGroup(ConnectsDesc c, TiesDesc t, std::tuple<Items...> items)
        : c_(std::move(c)), t_(std::move(t)), items_(std::move(items)) {}
    void setup() override {
        int seg = 0;
        bool barrier_next = false;
        segment_local_shared_.clear();
        std::apply([&](const auto&... it) { (add_item(it, seg, barrier_next), ...); }, items_);
        for (auto& [a, b] : c_.pairs) connect(a, b);
        for (auto& t : t_.entries) ties_.push_back(t);
    }
    void launch(detail::Runtime& rt) override;

private:
    ConnectsDesc c_;
    TiesDesc t_;
    std::tuple<Items...> items_;

    template <class T, class... A>
    void add_stage(const SubsystemDesc<T, A...>& d, int seg) {
        adopt(d.make(), d.name);
        stages_.push_back(static_cast<ComponentBase*>(children_.back().get()));
        stage_segment_.push_back(seg);
    }
    template <class T, class... A>
    void add_item(const SubsystemDesc<T, A...>& d, int& seg, bool& barrier_next) {
        open_segment(seg, barrier_next, false, false);
        add_stage(d, seg);
        ++seg;
    }
    template <class O, class... D>
    void add_item(const SegmentDesc<O, D...>& s, int& seg, bool& barrier_next) {
        open_segment(seg, barrier_next, detail::has_opt<local_mem::shared, O>::value,
                     detail::has_opt<range_mode::whole, O>::value);
        std::apply([&](const auto&... d) { (add_stage(d, seg), ...); }, s.descs);
        ++seg;
    }
    void add_item(const GlobalBarrierDesc&, int&, bool& barrier_next) { barrier_next = true; }
    void open_segment(int seg, bool& barrier_next, bool shared, bool whole) {
        segment_local_shared_.push_back(shared ? 1 : 0);
        segment_whole_.push_back(whole ? 1 : 0);
        segment_barrier_.push_back(barrier_next ? 1 : 0);
        barrier_next = false;
        (void)seg;
    }
};

template <class... Items>
struct FusedDesc {
    std::string name;
    ConnectsDesc connects;
    TiesDesc ties;
    std::tuple<Items...> items;
};

template <class Opts, class... Items>
struct FusedBuilder {
    std::string name;
    ConnectsDesc connects;
    TiesDesc ties;
    std::tuple<Items...> items;
    std::unique_ptr<Node> build() const { return std::make_unique<FusedGroup<Opts, Items...>>(connects, ties, items); }
};

namespace detail {
template <class Opts, class... Items>
FusedBuilder<Opts, Items...> make_fused(std::string name, ConnectsDesc c, TiesDesc t, Items... items) {
    return FusedBuilder<Opts, Items...>{std::move(name), std::move(c), std::move(t), std::tuple<Items...>(std::move(items)...)};
}
}  // namespace detail

namespace detail {
template <class... Items> inline constexpr bool leads_with_connects_v = false;
template <class I, class... R> inline constexpr bool leads_with_connects_v<I, R...> = std::is_same_v<I, ConnectsDesc>;
template <class... Items> inline constexpr bool leads_with_ties_v = false;
template <class I, class... R> inline constexpr bool leads_with_ties_v<I, R...> = std::is_same_v<I, TiesDesc>;
}  // namespace detail

/// fuse_components[<options>](name, [connects_desc(...)], [ties_desc(...)], items...): both descriptions are optional,
/// connects first (fused_component.hpp:524-569).
template <class... Opts, class... Items>
auto fuse_components(std::string name, ConnectsDesc c, TiesDesc t, Items... items) {
    return detail::make_fused<std::tuple<Opts...>>(std::move(name), std::move(c), std::move(t), std::move(items)...);
}
template <class... Opts, class... Items>
    requires(!detail::leads_with_ties_v<Items...>)
auto fuse_components(std::string name, ConnectsDesc c, Items... items) {
    return detail::make_fused<std::tuple<Opts...>>(std::move(name), std::move(c), TiesDesc{}, std::move(items)...);
}
template <class... Opts, class... Items>
    requires(!detail::leads_with_connects_v<Items...>)
auto fuse_components(std::string name, TiesDesc t, Items... items) {
    return detail::make_fused<std::tuple<Opts...>>(std::move(name), ConnectsDesc{}, std::move(t), std::move(items)...);
}
template <class... Opts, class... Items>
    requires(sizeof...(Items) >= 1 && !detail::leads_with_connects_v<Items...> && !detail::leads_with_ties_v<Items...>)
auto fuse_components(std::string name, Items... items) {
    return detail::make_fused<std::tuple<Opts...>>(std::move(name), ConnectsDesc{}, TiesDesc{}, std::move(items)...);
}

}  // namespace naga::cospan
