// naga/cospan/core.hpp — the data side of the cs:: API on the cspb runtime: dtypes, shapes, the device wrappers a
// component body indexes (Input, Output, Initializer), work-group items and local memory, launch descriptors, and
// initializer specifications.
//
// Mirrors the reference's dtype.hpp, metadata.hpp, wrappers.hpp, kernel.hpp (GroupItem :364-446, LocalMem :515-570,
// group functions :581-633) and init.hpp (fill :203-211, from_host :242-260, custom :269-296), so that component code
// written against the reference compiles unchanged (device functions need __host__ __device__ under nvcc; see
// cospanmdao_b200/annotate.py).
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <initializer_list>
#include <memory>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include <sycl/sycl.hpp>

namespace naga::slabkit {
class unordered_queue;
}

namespace naga::cospan {

namespace sk = naga::slabkit;

// ---- dtypes -----------------------------------------------------------------------------------------------------
enum class DType : std::uint8_t { f32, f64, i32, u32, i64, u64, u8, atomic_f32, atomic_i32, atomic_u32, atomic_u64 };

template <DType DT> struct cpp_type;
template <> struct cpp_type<DType::f32> { using type = float; };
template <> struct cpp_type<DType::f64> { using type = double; };
template <> struct cpp_type<DType::i32> { using type = std::int32_t; };
template <> struct cpp_type<DType::u32> { using type = std::uint32_t; };
template <> struct cpp_type<DType::i64> { using type = std::int64_t; };
template <> struct cpp_type<DType::u64> { using type = std::uint64_t; };
template <> struct cpp_type<DType::u8> { using type = std::uint8_t; };
template <> struct cpp_type<DType::atomic_f32> { using type = float; };
template <> struct cpp_type<DType::atomic_i32> { using type = std::int32_t; };
template <> struct cpp_type<DType::atomic_u32> { using type = std::uint32_t; };
template <> struct cpp_type<DType::atomic_u64> { using type = std::uint64_t; };
template <DType DT> using cpp_type_t = typename cpp_type<DT>::type;

constexpr bool is_atomic(DType d) {
    return d == DType::atomic_f32 || d == DType::atomic_i32 || d == DType::atomic_u32 || d == DType::atomic_u64;
}
template <DType DT> inline constexpr bool is_atomic_v = is_atomic(DT);
constexpr DType value_dtype(DType d) {
    switch (d) {
        case DType::atomic_f32: return DType::f32;
        case DType::atomic_i32: return DType::i32;
        case DType::atomic_u32: return DType::u32;
        case DType::atomic_u64: return DType::u64;
        default: return d;
    }
}
constexpr std::size_t dtype_size(DType d) {
    switch (value_dtype(d)) {
        case DType::f64: case DType::i64: case DType::u64: return 8;
        case DType::u8: return 1;
        default: return 4;
    }
}
constexpr bool dtype_compatible(DType a, DType b) { return value_dtype(a) == value_dtype(b); }
inline const char* dtype_name(DType d) {
    switch (d) {
        case DType::f32: return "f32"; case DType::f64: return "f64"; case DType::i32: return "i32";
        case DType::u32: return "u32"; case DType::i64: return "i64"; case DType::u64: return "u64";
        case DType::u8: return "u8"; case DType::atomic_f32: return "atomic_f32"; case DType::atomic_i32: return "atomic_i32";
        case DType::atomic_u32: return "atomic_u32"; case DType::atomic_u64: return "atomic_u64";
    }
    return "?";
}

// ---- shapes -----------------------------------------------------------------------------------------------------
struct Unspecified {};
inline constexpr Unspecified unspecified{};
template <int Rank>
constexpr std::array<Unspecified, Rank> unspecified_shape() { return {}; }

/// A declared or required shape: a rank and per-dimension extents, some possibly unknown.
struct ShapeSpec {
    int rank = -1;  // -1: nothing said
    std::array<std::size_t, 4> ext{};
    std::array<bool, 4> known{};
    bool empty() const { return rank < 0; }
};
namespace detail {
inline void put(ShapeSpec& s, int d, Unspecified) { s.known[d] = false; }
template <class T, class = std::enable_if_t<std::is_integral_v<T>>>
inline void put(ShapeSpec& s, int d, T v) {
    s.ext[d] = static_cast<std::size_t>(v);
    s.known[d] = true;
}
}  // namespace detail
template <class... S>
ShapeSpec shape(S... specs) {
    ShapeSpec s;
    s.rank = int(sizeof...(S));
    int d = 0;
    (detail::put(s, d++, specs), ...);
    return s;
}

/// The shape an initializer supplies: init::fill(v, {n, m}).
struct Shape {
    std::vector<std::size_t> ext;
    Shape(std::initializer_list<std::size_t> e) : ext(e) {}
    const Shape& get() const { return *this; }
    std::size_t elements() const {
        std::size_t n = 1;
        for (auto e : ext) n *= e;
        return n;
    }
};

// ---- device wrappers --------------------------------------------------------------------------------------------
namespace detail {
template <int R>
CS_HD inline std::size_t flat(const sycl::id<R>& i, const sycl::range<R>& stride) {
    std::size_t f = 0;
    for (int d = 0; d < R; ++d) f += i[d] * stride[d];
    return f;
}
}  // namespace detail

/// Input<DT, Rank>: a component's read-only view of a variable (data pointer, shape, row-major strides).
template <DType DT, int Rank>
struct Input {
    using value_type = cpp_type_t<DT>;
    static constexpr DType dtype = DT;
    static constexpr int rank = Rank;
    CS_HD sycl::range<Rank> shape() const { return shape_; }
    CS_HD std::size_t size() const { return shape_.size(); }
    CS_HD const value_type& operator[](const sycl::id<Rank>& i) const { return data_[detail::flat<Rank>(i, stride_)]; }
    template <int Q = Rank, class = std::enable_if_t<(Q > 1)>>
    CS_HD const value_type& operator[](std::size_t f) const { return data_[f]; }
    CS_HD const value_type* data() const { return data_; }

    sycl::range<Rank> shape_{};
    sycl::range<Rank> stride_{};
    const value_type* data_ = nullptr;
};

/// Output<DT, Rank>: a component's writable view. Atomic dtypes index as sycl::atomic_ref (relaxed, device scope).
template <DType DT, int Rank>
struct Output {
    using value_type = cpp_type_t<DT>;
    static constexpr DType dtype = DT;
    static constexpr int rank = Rank;
    CS_HD sycl::range<Rank> shape() const { return shape_; }
    CS_HD std::size_t size() const { return shape_.size(); }
    template <DType Q = DT, std::enable_if_t<!is_atomic_v<Q>, int> = 0>
    CS_HD value_type& operator[](const sycl::id<Rank>& i) const { return data_[detail::flat<Rank>(i, stride_)]; }
    template <DType Q = DT, std::enable_if_t<is_atomic_v<Q>, int> = 0>
    CS_HD sycl::atomic_ref<value_type> operator[](const sycl::id<Rank>& i) const {
        return sycl::atomic_ref<value_type>(data_[detail::flat<Rank>(i, stride_)]);
    }
    CS_HD value_type* data() const { return data_; }

    sycl::range<Rank> shape_{};
    sycl::range<Rank> stride_{};
    value_type* data_ = nullptr;
};

/// Initializer<DT, Rank>: what an init::custom function writes (a writable view, non-atomic indexing).
template <DType DT, int Rank>
struct Initializer {
    using value_type = cpp_type_t<DT>;
    CS_HD sycl::range<Rank> shape() const { return shape_; }
    CS_HD value_type& operator[](const sycl::id<Rank>& i) const { return data_[detail::flat<Rank>(i, stride_)]; }
    CS_HD value_type* data() const { return data_; }
    sycl::range<Rank> shape_{};
    sycl::range<Rank> stride_{};
    value_type* data_ = nullptr;
};

// ---- ragged ports (wrappers.hpp:236-347 of the reference) -------------------------------------------------------
// A ragged port is rank 2: N blocks, block i holding count(i) elements, the blocks stored end to end. The runtime
// keeps per-index extents and the N + 1 block offsets on the device: u32 (the reference's, so a ragged total is below
// 2^32), or u64 where the hook asked for them (counts_from<std::uint64_t>). A
// RaggedInput also reads a DENSE rank-2 variable, whose block i is row i.

/// Per-index counts given on the host, in a declaration: declare_output(m, "m", cs::counts({1, 0, 3})).
struct Counts {
    std::vector<std::size_t> v;
};
inline Counts counts(std::vector<std::size_t> v) { return Counts{std::move(v)}; }
/// The same as N + 1 block offsets (offsets[0] == 0, never decreasing).
struct Offsets {
    std::vector<std::size_t> v;
};
inline Offsets offsets(std::vector<std::size_t> v) {
    if (v.empty() || v[0] != 0)
        throw std::invalid_argument("naga::cospan: cs::offsets needs N + 1 >= 1 entries starting at 0");
    for (std::size_t i = 1; i < v.size(); ++i)
        if (v[i] < v[i - 1]) throw std::invalid_argument("naga::cospan: cs::offsets must not decrease");
    return Offsets{std::move(v)};
}
inline Counts counts_of(const Offsets& o) {
    Counts c;
    for (std::size_t i = 0; i + 1 < o.v.size(); ++i) c.v.push_back(o.v[i + 1] - o.v[i]);
    return c;
}

/// One block of a ragged port: a dense rank-1 view (`T` is const for an input).
template <class T, int R = 1>
struct Block {
    static_assert(R == 1, "naga::cospan: a ragged block has rank 1");
    CS_HD T& operator[](const sycl::id<1>& i) const { return data_[i[0]]; }
    CS_HD T& operator[](std::size_t f) const { return data_[f]; }
    CS_HD sycl::range<1> shape() const { return sycl::range<1>{n_}; }
    CS_HD std::size_t size() const { return n_; }
    T* data_ = nullptr;
    std::size_t n_ = 0;
};
/// The block of an atomic ragged output: indexing gives a relaxed device-scope atomic_ref.
template <class T, int R = 1>
struct AtomicBlock {
    CS_HD sycl::atomic_ref<T> operator[](const sycl::id<1>& i) const { return sycl::atomic_ref<T>(b_.data_[i[0]]); }
    CS_HD sycl::atomic_ref<T> operator[](std::size_t f) const { return sycl::atomic_ref<T>(b_.data_[f]); }
    CS_HD sycl::range<1> shape() const { return b_.shape(); }
    CS_HD std::size_t size() const { return b_.size(); }
    Block<T, R> b_;
};

namespace detail {
/// Block i: extents from the per-index array (a ragged variable) or the row length (a dense one); the start from the
/// block offsets, or i rows in.
template <class T>
CS_HD inline Block<T> ragged_block(T* data, const std::uint32_t* offs, const std::uint64_t* offs64,
                                   const std::uint32_t* ext, std::size_t row, std::size_t i) {
    Block<T> b;
    b.n_ = ext ? std::size_t(ext[i]) : row;
    b.data_ = data + (offs64 ? std::size_t(offs64[i]) : offs ? std::size_t(offs[i]) : i * row);
    return b;
}
}  // namespace detail

/// RaggedInput<DT, 2>: a read-only ragged port. size() is N; block(i) is block i.
template <DType DT, int Rank>
struct RaggedInput {
    static_assert(Rank == 2, "naga::cospan: a ragged port is rank 2");
    static_assert(!is_atomic_v<DT>, "naga::cospan: a ragged input is not atomic");
    using value_type = cpp_type_t<DT>;
    static constexpr DType dtype = DT;
    static constexpr int rank = Rank;
    static constexpr bool ragged = true;
    CS_HD std::size_t size() const { return n_; }
    CS_HD Block<const value_type> block(std::size_t i) const { return detail::ragged_block(data_, offs_, offs64_, ext_, row_, i); }

    std::size_t n_ = 0;
    const value_type* data_ = nullptr;
    const std::uint32_t* offs_ = nullptr;
    const std::uint64_t* offs64_ = nullptr;  // a column with u64 offsets (counts_from<std::uint64_t>)
    const std::uint32_t* ext_ = nullptr;
    std::size_t row_ = 0;
};

/// RaggedOutput<DT, 2>: the writable twin; with an atomic dtype, block(i) is an AtomicBlock.
template <DType DT, int Rank>
struct RaggedOutput {
    static_assert(Rank == 2, "naga::cospan: a ragged port is rank 2");
    using value_type = cpp_type_t<DT>;
    static constexpr DType dtype = DT;
    static constexpr int rank = Rank;
    static constexpr bool ragged = true;
    CS_HD std::size_t size() const { return n_; }
    template <DType Q = DT, std::enable_if_t<!is_atomic_v<Q>, int> = 0>
    CS_HD Block<value_type> block(std::size_t i) const { return detail::ragged_block(data_, offs_, offs64_, ext_, row_, i); }
    template <DType Q = DT, std::enable_if_t<is_atomic_v<Q>, int> = 0>
    CS_HD AtomicBlock<value_type> block(std::size_t i) const {
        return AtomicBlock<value_type>{detail::ragged_block(data_, offs_, offs64_, ext_, row_, i)};
    }

    std::size_t n_ = 0;
    value_type* data_ = nullptr;
    const std::uint32_t* offs_ = nullptr;
    const std::uint64_t* offs64_ = nullptr;  // a column with u64 offsets (counts_from<std::uint64_t>)
    const std::uint32_t* ext_ = nullptr;
    std::size_t row_ = 0;
};

static_assert(std::is_trivially_copyable_v<RaggedInput<DType::f32, 2>>);
static_assert(std::is_trivially_copyable_v<RaggedOutput<DType::atomic_f32, 2>>);

namespace detail {
struct Column;  // the device counts and offsets of a ragged variable (model.hpp)
}

/// The shape of a ragged port, as a component's shape_of returns it and its set_shape takes it (component.hpp:
/// 130-160 of the reference): N, the total, and the counts — on the host (`counts`) or on the device (`column`).
struct RaggedShape {
    std::size_t n = 0;
    std::uint64_t total = 0;
    std::vector<std::size_t> counts;
    std::shared_ptr<const detail::Column> column;
    std::uint64_t column_version = 0;
    bool on_device() const noexcept { return column != nullptr; }
};

// ---- work-group items -------------------------------------------------------------------------------------------
template <int R>
struct Group {
    sycl::id<R> gid;
    sycl::range<R> grange;
    sycl::range<R> local;
    CS_HD sycl::group<3> to_sycl() const {
        sycl::group<3> g;
        for (int d = 0; d < 3; ++d) {
            g.local[d] = d < 3 - R ? 1 : local[d - (3 - R)];
            g.grange[d] = d < 3 - R ? 1 : grange[d - (3 - R)];
            g.gid[d] = d < 3 - R ? 0 : gid[d - (3 - R)];
        }
        return g;
    }
    CS_HD operator sycl::group<3>() const { return to_sycl(); }
    CS_HD std::size_t get_local_linear_id() const { return sycl::detail::thread_x(); }
    CS_HD sycl::range<R> get_local_range() const { return local; }
    CS_HD sycl::id<R> get_group_id() const { return gid; }
    CS_HD sycl::range<R> get_group_range() const { return grange; }
};

/// What a group-range body receives: the sycl::nd_item API over the stage's rank-R ids (kernel.hpp:364-446). Group ids
/// count within the stage's segment; local ids are the work-item's place in its work-group (row-major).
template <int R>
struct GroupItem {
    sycl::id<R> group_id;
    sycl::range<R> group_range;
    sycl::range<R> local_range;
    std::uint32_t segment = 0, segments = 1;

    CS_HD sycl::id<R> get_local_id() const {
        sycl::id<R> r;
        std::size_t l = sycl::detail::thread_x();
        for (int d = R - 1; d >= 0; --d) {
            r[d] = l % local_range[d];
            l /= local_range[d];
        }
        return r;
    }
    CS_HD std::size_t get_local_id(int d) const { return get_local_id()[d]; }
    CS_HD sycl::range<R> get_local_range() const { return local_range; }
    CS_HD std::size_t get_local_range(int d) const { return local_range[d]; }
    CS_HD std::size_t get_local_linear_id() const { return sycl::detail::thread_x(); }
    CS_HD sycl::id<R> get_group_id() const { return group_id; }
    CS_HD std::size_t get_group(int d) const { return group_id[d]; }
    CS_HD Group<R> get_group() const { return Group<R>{group_id, group_range, local_range}; }
    CS_HD sycl::range<R> get_group_range() const { return group_range; }
    CS_HD std::size_t get_group_range(int d) const { return group_range[d]; }
    CS_HD std::size_t get_group_linear_id() const {
        std::size_t l = 0;
        for (int d = 0; d < R; ++d) l = l * group_range[d] + group_id[d];
        return l;
    }
    CS_HD std::size_t get_global_id(int d) const { return group_id[d] * local_range[d] + get_local_id(d); }
    CS_HD sycl::id<R> get_global_id() const {
        sycl::id<R> g;
        const sycl::id<R> l = get_local_id();
        for (int d = 0; d < R; ++d) g[d] = group_id[d] * local_range[d] + l[d];
        return g;
    }
    CS_HD sycl::range<R> get_global_range() const {
        sycl::range<R> g;
        for (int d = 0; d < R; ++d) g[d] = group_range[d] * local_range[d];
        return g;
    }
    CS_HD std::size_t get_global_linear_id() const {
        const sycl::id<R> g = get_global_id();
        const sycl::range<R> r = get_global_range();
        std::size_t l = 0;
        for (int d = 0; d < R; ++d) l = l * r[d] + g[d];
        return l;
    }
    CS_HD std::size_t get_segment() const { return segment; }
    CS_HD std::size_t get_segment_count() const { return segments; }
    /// Waits for group g of an earlier segment. This backend runs the segments of a fused group one after the other
    /// with a grid barrier between them, so every group of an earlier segment has finished: nothing to wait for.
    CS_HD void wait_group(std::size_t, const sycl::id<R>&) const { sycl::detail::sync_block(); }
    CS_HD void wait_earlier_segments() const { sycl::detail::sync_block(); }
    CS_HD sycl::nd_item<3> to_sycl() const {
        sycl::nd_item<3> it;
        it.g = get_group().to_sycl();
        return it;
    }
};

template <int R>
CS_HD inline void group_barrier(const Group<R>&) { sycl::detail::sync_block(); }
template <int R, class T, class Op>
CS_HD inline T reduce_over_group(const Group<R>& g, T x, Op op) {
    return sycl::reduce_over_group(sycl::group<3>{}, x, op);
}
template <int R, class T>
CS_HD inline T group_broadcast(const Group<R>&, T x, std::size_t id = 0) {
    return sycl::group_broadcast(sycl::group<3>{}, x, id);
}

// ---- local memory -----------------------------------------------------------------------------------------------
template <DType DT, int Rank>
struct LocalView {
    using value_type = cpp_type_t<DT>;
    CS_HD LocalView(value_type* d, sycl::range<Rank> s) : data_(d), shape_(s) {}
    CS_HD value_type& operator[](const sycl::id<Rank>& idx) const {
        std::size_t f = 0;
        for (int d = 0; d < Rank; ++d) f = f * shape_[d] + idx[d];
        return data_[f];
    }
    template <int Q = Rank, class = std::enable_if_t<(Q > 1)>>
    CS_HD value_type& operator[](std::size_t f) const { return data_[f]; }
    CS_HD sycl::range<Rank> shape() const { return shape_; }
    CS_HD std::size_t size() const { return shape_.size(); }
    value_type* data_;
    sycl::range<Rank> shape_;
};

template <DType DT, int Rank>
struct LocalArray {
    using value_type = cpp_type_t<DT>;
    using view_type = LocalView<DT, Rank>;
    static constexpr DType dtype = DT;
    static constexpr int rank = Rank;
};

/// LocalViews<V...>: what LocalMem::get returns, the views in declaration order. A tuple-like type of its own (std::tuple
/// is host-only code under nvcc) that structured bindings unpack: auto [a, b] = lm.get(it).
namespace detail {
template <std::size_t I, class T>
struct ViewSlot {
    T v;
};
template <class Seq, class... V> struct ViewPack;
template <std::size_t... I, class... V>
struct ViewPack<std::index_sequence<I...>, V...> : ViewSlot<I, V>... {
    CS_HD explicit ViewPack(V... v) : ViewSlot<I, V>{v}... {}
};
template <std::size_t I, class T>
CS_HD T& slot_ref(ViewSlot<I, T>& s) { return s.v; }
template <std::size_t I, class T>
CS_HD const T& slot_cref(const ViewSlot<I, T>& s) { return s.v; }
}  // namespace detail

template <class... V>
struct LocalViews : detail::ViewPack<std::index_sequence_for<V...>, V...> {
    CS_HD explicit LocalViews(V... v) : detail::ViewPack<std::index_sequence_for<V...>, V...>(v...) {}
    template <std::size_t I> CS_HD auto& get() & { return detail::slot_ref<I>(*this); }
    template <std::size_t I> CS_HD const auto& get() const& { return detail::slot_cref<I>(*this); }
    template <std::size_t I> CS_HD auto&& get() && {
        auto& r = detail::slot_ref<I>(*this);
        return static_cast<std::remove_reference_t<decltype(r)>&&>(r);
    }
};

/// LocalMem<Arrays...>: a group-range stage's local memory (kernel.hpp:515-570). get(it) returns the views of its
/// arrays, in declaration order (LocalViews, for structured bindings). The runtime fills base and shapes.
template <class... Arrays>
struct LocalMem {
    unsigned char* base = nullptr;
    std::array<std::array<std::size_t, 3>, sizeof...(Arrays)> shapes{};
    std::array<std::size_t, sizeof...(Arrays)> offsets{};

    template <int R>
    CS_HD auto get(const GroupItem<R>&) const { return views(std::index_sequence_for<Arrays...>{}); }

private:
    template <std::size_t... I>
    CS_HD LocalViews<typename Arrays::view_type...> views(std::index_sequence<I...>) const {
        return LocalViews<typename Arrays::view_type...>(view<Arrays>(I)...);
    }
    template <class A>
    CS_HD typename A::view_type view(std::size_t i) const {
        sycl::range<A::rank> r;
        for (int d = 0; d < A::rank; ++d) r[d] = shapes[i][d];
        return typename A::view_type(reinterpret_cast<typename A::value_type*>(base + offsets[i]), r);
    }
};

namespace detail {
template <class T> struct is_local_mem : std::false_type {};
template <class... A> struct is_local_mem<LocalMem<A...>> : std::true_type {};
template <class T> struct local_arrays;
template <class... A> struct local_arrays<LocalMem<A...>> {
    static constexpr std::size_t count = sizeof...(A);
    static std::array<std::size_t, sizeof...(A)> elem_sizes() { return {sizeof(typename A::value_type)...}; }
    static std::array<int, sizeof...(A)> ranks() { return {A::rank...}; }
};
}  // namespace detail

// ---- launch descriptors -----------------------------------------------------------------------------------------
struct LaunchDescription {
    int rank = 0;
    std::array<std::size_t, 3> range{1, 1, 1};
    bool has_wg = false;
    std::array<std::size_t, 3> wg{1, 1, 1};
    std::vector<std::array<std::size_t, 3>> local;  // one shape per local array
    std::vector<int> local_ranks;
    virtual ~LaunchDescription() = default;
};
template <int R> struct RangeDesc { sycl::range<R> r; };
template <int R> struct WgDesc { sycl::range<R> r; };
struct LocalDesc {
    std::vector<std::array<std::size_t, 3>> shapes;
    std::vector<int> ranks;
};
template <int R> RangeDesc<R> range_desc(sycl::range<R> r) { return {r}; }
template <int R> WgDesc<R> wg_desc(sycl::range<R> r) { return {r}; }
namespace detail {
template <int R>
std::array<std::size_t, 3> to3(const sycl::range<R>& r) {
    std::array<std::size_t, 3> a{1, 1, 1};
    for (int k = 0; k < R; ++k) a[k] = r[k];
    return a;
}
}  // namespace detail
template <int... R>
LocalDesc local_desc(sycl::range<R>... rs) {
    LocalDesc d;
    (d.shapes.push_back(detail::to3<R>(rs)), ...);
    (d.ranks.push_back(R), ...);
    return d;
}

// ---- initializers -----------------------------------------------------------------------------------------------
namespace detail {
struct InitTarget;  // defined by the runtime
}
/// What an initializer does to a variable when it is (re)initialized: a function of the target, plus the shape it
/// supplies (if any).
struct InitSpec {
    std::function<void(detail::InitTarget&)> run;
    std::optional<std::vector<std::size_t>> shape;  // extents this initializer supplies
    std::optional<std::size_t> flat;                // from_host without a shape: its element count
    std::optional<double> scalar;                   // a fill value (lets the runtime read a scale on the host)
};

template <DType DT, int Rank>
using CustomFn = std::function<sycl::event(sk::unordered_queue&, const sycl::device&, const std::vector<sycl::event>&,
                                           Initializer<DT, Rank>)>;

}  // namespace naga::cospan

template <class... V>
struct std::tuple_size<naga::cospan::LocalViews<V...>> : std::integral_constant<std::size_t, sizeof...(V)> {};
template <std::size_t I, class... V>
struct std::tuple_element<I, naga::cospan::LocalViews<V...>> {
    using type = std::tuple_element_t<I, std::tuple<V...>>;
};
