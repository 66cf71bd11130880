// Ragged ports and ragged shape hooks of the cs:: runtime, every case through a cs::Model on the GPU (compiled by
// cospanmdao_b200.examples.build_runtime_tests, run by tests/test_examples_gpu.py). The cases follow the behaviour the
// reference's tests/test_ragged.cpp describes:
//   - a counts_from hook builds a ragged shape on the device (cspb_build_column) and a chain of ragged components
//     follows it over forwards whose counts change (empty blocks, growth, shrinking, all empty, N = 0);
//   - counts_from reads column 0 of a rank-2 source; offsets_from takes N + 1 offsets;
//   - declared counts meet at a connect (equal: fine; different N or counts: an error in setup);
//   - a RaggedInput reads a dense rank-2 port as rows;
//   - a hook on a ragged OUTPUT owns its shape, over growing and shrinking counts;
//   - errors: a dense Input on a ragged source, negative counts, totals past 2^32 - 1, bad offsets, dense views of a
//     ragged variable, views of the wrong dtype.
// Beyond the reference (which refuses ragged ports in fused groups): a fused group of an index-range stage that writes
// a ragged output and a work-group stage that reduces each block must give the unfused result.
// Prints one line per case and "ALL OK" when every case passes; exits 1 otherwise.
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "naga/cospan/cospan.hpp"

namespace cs = naga::cospan;
using cs::DType;
using Sizes = std::vector<std::size_t>;

namespace rg {

int g_fails = 0;

void check(bool ok, const std::string& what) {
    if (!ok) {
        std::printf("  FAIL: %s\n", what.c_str());
        ++g_fails;
    }
}

template <class F>
void expect_error(F&& f, const std::vector<std::string>& needles, const std::string& what) {
    std::string msg = "<no exception>";
    try {
        f();
    } catch (const std::exception& e) {
        msg = e.what();
    }
    for (const auto& n : needles)
        if (msg.find(n) == std::string::npos) {
            std::printf("  FAIL: %s: \"%s\" not in: %s\n", what.c_str(), n.c_str(), msg.c_str());
            ++g_fails;
        }
}

// ---- components ---------------------------------------------------------------------------------------------------

// counts[i] = raw[i]; N fixed by the declaration of raw
class CopyCounts : public cs::Component<CopyCounts> {
public:
    struct Inputs { cs::Input<DType::u32, 1> raw; };
    struct Outputs { cs::Output<DType::u32, 1> counts; };
    __host__ __device__ static void compute_forward(sycl::id<1> i, const Inputs& in, const Outputs& out) {
        out.counts[i] = in.raw[i];
    }
    Inputs inputs;
    Outputs outputs;
    explicit CopyCounts(std::size_t n) : n_{n} {}
    void declare() override {
        declare_input(inputs.raw, "raw", n_);
        declare_output(outputs.counts, "counts", cs::unspecified);
    }
    void prepare_forward() override { set_shape(outputs.counts, shape_of(inputs.raw)[0]); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(outputs.counts.shape()));
    }

private:
    std::size_t n_;
};

// pts takes the shape of the hooked layout; pts.block(i)[j] = i * 1000 + j
class FillBlocks : public cs::Component<FillBlocks> {
public:
    struct Inputs { cs::RaggedInput<DType::f32, 2> layout; };
    struct Outputs { cs::RaggedOutput<DType::f32, 2> pts; };
    __host__ __device__ static void compute_forward(sycl::id<1> id, const Inputs&, const Outputs& out) {
        const std::size_t i = id[0];
        auto b = out.pts.block(i);
        for (std::size_t j = 0; j < b.shape()[0]; ++j) b[j] = static_cast<float>(i * 1000 + j);
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.layout, "layout");
        declare_output(outputs.pts, "pts");
    }
    void prepare_forward() override { set_shape(outputs.pts, shape_of(inputs.layout)); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(sycl::range<1>{inputs.layout.size()}));
    }
};

// out = 2 in, block by block; out takes the shape of in
class Twice : public cs::Component<Twice> {
public:
    struct Inputs { cs::RaggedInput<DType::f32, 2> in; };
    struct Outputs { cs::RaggedOutput<DType::f32, 2> out; };
    __host__ __device__ static void compute_forward(sycl::id<1> id, const Inputs& in, const Outputs& out) {
        auto bi = in.in.block(id[0]);
        auto bo = out.out.block(id[0]);
        for (std::size_t q = 0; q < bi.size(); ++q) bo[q] = 2.0f * bi[q];
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.in, "in");
        declare_output(outputs.out, "out");
    }
    void prepare_forward() override { set_shape(outputs.out, shape_of(inputs.in)); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(sycl::range<1>{inputs.in.size()}));
    }
};

// sums[i] = the sum of block i, in order
class BlockSums : public cs::Component<BlockSums> {
public:
    struct Inputs { cs::RaggedInput<DType::f32, 2> pts; };
    struct Outputs { cs::Output<DType::f32, 1> sums; };
    __host__ __device__ static void compute_forward(sycl::id<1> id, const Inputs& in, const Outputs& out) {
        auto b = in.pts.block(id[0]);
        float s = 0.0f;
        for (std::size_t q = 0; q < b.size(); ++q) s += b[q];
        out.sums[id] = s;
    }
    Inputs inputs;
    Outputs outputs;
    BlockSums() = default;
    explicit BlockSums(Sizes declared) : declared_{std::move(declared)}, has_{true} {}
    void declare() override {
        if (has_) declare_input(inputs.pts, "pts", cs::counts(declared_));
        else declare_input(inputs.pts, "pts");
        declare_output(outputs.sums, "sums", cs::unspecified);
    }
    void prepare_forward() override { set_shape(outputs.sums, shape_of(inputs.pts).n); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(outputs.sums.shape()));
    }

private:
    Sizes declared_;
    bool has_ = false;
};

// the same sums by work-groups of 64: group g reduces block g
class GroupBlockSums : public cs::Component<GroupBlockSums> {
public:
    static constexpr std::size_t kWg = 64;
    struct Inputs { cs::RaggedInput<DType::f32, 2> pts; };
    struct Outputs { cs::Output<DType::f32, 1> sums; };
    __host__ __device__ static void compute_forward(cs::GroupItem<1> it, const Inputs& in, const Outputs& out) {
        const std::size_t g = it.get_group(0), l = it.get_local_id(0);
        auto b = in.pts.block(g);
        float s = 0.0f;
        for (std::size_t q = l; q < b.size(); q += kWg) s += b[q];
        const float t = cs::reduce_over_group(it.get_group(), s, sycl::plus<float>());
        if (l == 0) out.sums[sycl::id<1>{g}] = t;
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.pts, "pts");
        declare_output(outputs.sums, "sums", cs::unspecified);
    }
    void prepare_forward() override { set_shape(outputs.sums, shape_of(inputs.pts).n); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(sycl::range<1>{inputs.pts.size() * kWg}), cs::wg_desc(sycl::range<1>{kWg}));
    }
};

// a ragged output with declared counts; m.block(i)[j] = i * 100 + j
class Maker : public cs::Component<Maker> {
public:
    struct Inputs {};
    struct Outputs { cs::RaggedOutput<DType::f32, 2> m; };
    __host__ __device__ static void compute_forward(sycl::id<1> id, const Inputs&, const Outputs& out) {
        const std::size_t i = id[0];
        auto b = out.m.block(i);
        for (std::size_t j = 0; j < b.size(); ++j) b[j] = static_cast<float>(i * 100 + j);
    }
    Inputs inputs;
    Outputs outputs;
    explicit Maker(Sizes sizes) : sizes_{std::move(sizes)} {}
    void declare() override { declare_output(outputs.m, "m", cs::counts(sizes_)); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(sycl::range<1>{sizes_.size()}));
    }

private:
    Sizes sizes_;
};

// a ragged layout hooked from the counts in `cnt` (dtype DT, rank R); v takes its shape; v.block(i)[j] = i * 100 + j
template <DType DT, int R>
class FromCounts : public cs::Component<FromCounts<DT, R>> {
public:
    struct Inputs {
        cs::Input<DT, R> cnt;
        cs::RaggedInput<DType::f32, 2> layout;
    };
    struct Outputs { cs::RaggedOutput<DType::f32, 2> v; };
    __host__ __device__ static void compute_forward(sycl::id<1> id, const Inputs&, const Outputs& out) {
        const std::size_t i = id[0];
        auto b = out.v.block(i);
        for (std::size_t j = 0; j < b.size(); ++j) b[j] = static_cast<float>(i * 100 + j);
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        if constexpr (R == 2) this->declare_input(inputs.cnt, "cnt", cs::unspecified, cs::unspecified);
        else this->declare_input(inputs.cnt, "cnt", cs::unspecified);
        this->declare_input(inputs.layout, "layout");
        this->declare_output(outputs.v, "v");
    }
    void prepare_forward() override { this->set_shape(outputs.v, this->shape_of(inputs.layout)); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return this->create_launch_config(cs::range_desc(sycl::range<1>{inputs.layout.size()}));
    }
};

// a ragged OUTPUT whose shape a hook owns (no set_shape); v.block(i)[j] = i * 100 + j
class HookedOut : public cs::Component<HookedOut> {
public:
    struct Inputs { cs::Input<DType::u32, 1> cnt; };
    struct Outputs { cs::RaggedOutput<DType::f32, 2> v; };
    __host__ __device__ static void compute_forward(sycl::id<1> id, const Inputs&, const Outputs& out) {
        const std::size_t i = id[0];
        auto b = out.v.block(i);
        for (std::size_t j = 0; j < b.size(); ++j) b[j] = static_cast<float>(i * 100 + j);
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.cnt, "cnt", cs::unspecified);
        declare_output(outputs.v, "v");
    }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(sycl::range<1>{inputs.cnt.shape()[0]}));
    }
};

// a dense rank-2 output: d[i][j] = 10 i + j
class DenseRows : public cs::Component<DenseRows> {
public:
    struct Inputs {};
    struct Outputs { cs::Output<DType::f32, 2> d; };
    __host__ __device__ static void compute_forward(sycl::id<2> i, const Inputs&, const Outputs& out) {
        out.d[i] = static_cast<float>(i[0] * 10 + i[1]);
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override { declare_output(outputs.d, "d", 3, 4); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(outputs.d.shape()));
    }
};

// a dense input (would take a ragged source through unspecified dimensions)
class DenseIn : public cs::Component<DenseIn> {
public:
    struct Inputs { cs::Input<DType::f32, 2> in; };
    struct Outputs {};
    __host__ __device__ static void compute_forward(sycl::id<1>, const Inputs&, const Outputs&) {}
    Inputs inputs;
    Outputs outputs;
    void declare() override { declare_input(inputs.in, "in", cs::unspecified, cs::unspecified); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(sycl::range<1>{4}));
    }
};

// ---- systems ------------------------------------------------------------------------------------------------------

class Chain : public cs::System {
    std::size_t n_;

public:
    explicit Chain(std::size_t n) : n_{n} {}
    void setup() override {
        add_subsystem(cs::subsystem_desc<CopyCounts>("counts", n_));
        add_subsystem(cs::subsystem_desc<FillBlocks>("fill"));
        add_subsystem(cs::subsystem_desc<Twice>("scale"));
        add_subsystem(cs::subsystem_desc<BlockSums>("sum"));
        shape_hook("fill.layout", cs::ragged::counts_from("counts.counts"));
        connect("fill.pts", "scale.in");
        connect("scale.out", "sum.pts");
    }
};

template <class C, bool Offsets = false>
class HookedOn : public cs::System {
public:
    void setup() override {
        add_subsystem(cs::subsystem_desc<C>("c"));
        if constexpr (Offsets) shape_hook("c.layout", cs::ragged::offsets_from("c.cnt"));
        else shape_hook("c.layout", cs::ragged::counts_from("c.cnt"));
    }
};

class HookedOutTop : public cs::System {
public:
    void setup() override {
        add_subsystem(cs::subsystem_desc<HookedOut>("c"));
        shape_hook("c.v", cs::ragged::counts_from("c.cnt"));
    }
};

class MakeTake : public cs::System {
    Sizes make_, take_;

public:
    MakeTake(Sizes m, Sizes t) : make_{std::move(m)}, take_{std::move(t)} {}
    void setup() override {
        add_subsystem(cs::subsystem_desc<Maker>("make", make_));
        add_subsystem(cs::subsystem_desc<BlockSums>("take", take_));
        connect("make.m", "take.pts");
    }
};

class DenseTop : public cs::System {
public:
    void setup() override {
        add_subsystem(cs::subsystem_desc<DenseRows>("gen"));
        add_subsystem(cs::subsystem_desc<BlockSums>("sum"));
        connect("gen.d", "sum.pts");
    }
};

class DenseOnRagged : public cs::System {
public:
    void setup() override {
        add_subsystem(cs::subsystem_desc<Maker>("make", Sizes{1, 0, 3, 2}));
        add_subsystem(cs::subsystem_desc<DenseIn>("c"));
        connect("make.m", "c.in");
    }
};

// fused: an index-range stage writes the ragged output, a barrier, then a work-group stage (and an index-range
// stage) reduce it
class FusedRagged : public cs::System {
    Sizes sizes_;

public:
    explicit FusedRagged(Sizes s) : sizes_{std::move(s)} {}
    void setup() override {
        add_subsystem(cs::fuse_components(
            "w", cs::connects_desc({{"make.m", "gsum.pts"}, {"make.m", "isum.pts"}}),
            cs::subsystem_desc<Maker>("make", sizes_), cs::global_barrier(), cs::subsystem_desc<GroupBlockSums>("gsum"),
            cs::global_barrier(), cs::subsystem_desc<BlockSums>("isum")));
    }
};
class UnfusedRagged : public cs::System {
    Sizes sizes_;

public:
    explicit UnfusedRagged(Sizes s) : sizes_{std::move(s)} {}
    void setup() override {
        add_subsystem(cs::subsystem_desc<Maker>("make", sizes_));
        add_subsystem(cs::subsystem_desc<GroupBlockSums>("gsum"));
        connect("make.m", "gsum.pts");
    }
};

// ---- host references ------------------------------------------------------------------------------------------------

struct Flat {
    std::vector<float> data;
    std::vector<std::uint64_t> offsets{0};
};
template <class C>
Flat blocks_of(const std::vector<C>& counts, std::size_t mul) {
    Flat f;
    for (std::size_t i = 0; i < counts.size(); ++i) {
        for (std::size_t j = 0; j < std::size_t(counts[i]); ++j) f.data.push_back(static_cast<float>(i * mul + j));
        f.offsets.push_back(f.data.size());
    }
    return f;
}
template <class V>
std::vector<float> flat_of(const V& v) {
    return std::vector<float>(v.span().begin(), v.span().end());
}
template <class V>
void check_ragged(const V& v, const Flat& want, const std::string& what) {
    check(v.n() + 1 == want.offsets.size(), what + ": n");
    check(v.block_offsets() == want.offsets, what + ": block offsets");
    check(flat_of(v) == want.data, what + ": data");
    for (std::size_t i = 0; i + 1 < want.offsets.size() && i < v.n(); ++i)
        check(v.block(i).size() == want.offsets[i + 1] - want.offsets[i], what + ": block " + std::to_string(i) + " size");
}

// ---- cases ----------------------------------------------------------------------------------------------------------

void chain_forward(cs::Model& m, const std::vector<std::uint32_t>& counts) {
    const std::string tag = "counts of size " + std::to_string(counts.size());
    if (!counts.empty()) m.update_input("counts.raw", cs::init::from_host(counts));
    m.run();
    m.wait();
    const Flat ref = blocks_of(counts, 1000);
    auto sums = m.view_output<DType::f32, 1>("sum.sums");
    sums.sync();
    check(sums.span().size() == counts.size(), tag + ": sums size");
    for (std::size_t i = 0; i < counts.size() && i < sums.span().size(); ++i) {
        float want = 0.0f;
        for (std::uint64_t q = ref.offsets[i]; q < ref.offsets[i + 1]; ++q) want += 2.0f * ref.data[q];
        check(sums.span()[i] == want, tag + ": sum of block " + std::to_string(i));
    }
    auto pts = m.view_ragged_output<DType::f32, 2>("fill.pts");
    pts.sync();
    check_ragged(pts, ref, tag + ": fill.pts");
    for (std::size_t i = 0; i < counts.size(); ++i)
        for (std::size_t j = 0; j < counts[i] && j < pts.block(i).size(); ++j)
            check(pts.block(i)[j] == static_cast<float>(i * 1000 + j), tag + ": fill.pts element");
    Flat twice = ref;
    for (auto& x : twice.data) x *= 2.0f;
    auto scaled = m.view_ragged_output<DType::f32, 2>("scale.out");
    scaled.sync();
    check_ragged(scaled, twice, tag + ": scale.out");
    auto peer = m.view_ragged_input<DType::f32, 2>("scale.in");
    peer.sync();
    check_ragged(peer, ref, tag + ": scale.in");
}

void case_chain() {
    cs::Model m = cs::create_model<Chain>(std::size_t{6});
    m.setup();
    chain_forward(m, {3, 0, 2, 4, 0, 1});  // an empty block in the middle, one at the end
    chain_forward(m, {0, 5, 1, 0, 2, 2});  // an empty first block
    chain_forward(m, {1, 0, 0, 0, 0, 0});  // shrinks
    chain_forward(m, {0, 0, 0, 0, 0, 0});  // every block empty
    chain_forward(m, {2, 2, 2, 2, 2, 7});  // grows back
    // and wider: 5000 blocks of up to 300 elements (the column reallocates)
    cs::Model big = cs::create_model<Chain>(std::size_t{5000});
    big.setup();
    std::vector<std::uint32_t> c(5000);
    for (std::size_t i = 0; i < c.size(); ++i) c[i] = std::uint32_t((i * 7919u) % 301u);
    chain_forward(big, c);
}

void case_zero_blocks() {
    cs::Model m = cs::create_model<Chain>(std::size_t{0});
    m.setup();
    chain_forward(m, {});
    auto pts = m.view_ragged_output<DType::f32, 2>("fill.pts");
    pts.sync();
    check(pts.n() == 0 && pts.block_offsets() == std::vector<std::uint64_t>{0} && pts.size() == 0, "N = 0");
}

void case_column0() {
    cs::Model m = cs::create_model<HookedOn<FromCounts<DType::u32, 2>>>();
    m.setup();
    m.update_input("c.cnt", cs::init::from_host(std::vector<std::uint32_t>{2, 9, 0, 9, 3, 9, 1, 9}, cs::Shape{4, 2}));
    m.run();
    m.wait();
    auto v = m.view_ragged_output<DType::f32, 2>("c.v");
    v.sync();
    check(v.n() == 4, "column 0: n");
    check(v.block_offsets() == std::vector<std::uint64_t>{0, 2, 2, 5, 6}, "column 0: offsets");
    check(flat_of(v) == std::vector<float>{0, 1, 200, 201, 202, 300}, "column 0: data");
}

void case_offsets_from() {
    cs::Model m = cs::create_model<HookedOn<FromCounts<DType::i64, 1>, true>>();
    m.setup();
    m.update_input("c.cnt", cs::init::from_host(std::vector<std::int64_t>{0, 3, 3, 4, 8}));
    m.run();
    m.wait();
    auto v = m.view_ragged_output<DType::f32, 2>("c.v");
    v.sync();
    check_ragged(v, blocks_of(std::vector<int>{3, 0, 1, 4}, 100), "offsets_from");
    // offsets that do not start at 0, or decrease, are an error of the hook
    m.update_input("c.cnt", cs::init::from_host(std::vector<std::int64_t>{1, 3, 4}));
    expect_error([&] { m.run(); }, {"shape hook on 'c.layout'", "do not start at 0, or decrease"}, "offsets from 1");
    m.wait();
    m.update_input("c.cnt", cs::init::from_host(std::vector<std::int64_t>{0, 3, 2}));
    expect_error([&] { m.run(); }, {"shape hook on 'c.layout'", "do not start at 0, or decrease"}, "decreasing offsets");
    m.wait();
}

void case_declared_counts() {
    const Sizes sizes{1, 0, 3, 2};
    cs::Model m = cs::create_model<MakeTake>(sizes, sizes);
    m.setup();
    m.run();
    m.wait();
    auto sums = m.view_output<DType::f32, 1>("take.sums");
    sums.sync();
    for (std::size_t i = 0; i < sizes.size(); ++i) {
        float want = 0.0f;
        for (std::size_t j = 0; j < sizes[i]; ++j) want += static_cast<float>(i * 100 + j);
        check(sums.span().size() == 4 && sums.span()[i] == want, "declared counts: sum " + std::to_string(i));
    }
    auto mm = m.view_ragged_output<DType::f32, 2>("make.m");
    mm.sync();
    check_ragged(mm, blocks_of(sizes, 100), "declared counts: make.m");
    cs::Model zero = cs::create_model<MakeTake>(Sizes{}, Sizes{});
    zero.setup();
    zero.run();
    zero.wait();
    auto z = zero.view_ragged_output<DType::f32, 2>("make.m");
    z.sync();
    check(z.n() == 0 && z.block_offsets() == std::vector<std::uint64_t>{0}, "declared counts: N = 0");
}

void case_declared_mismatch() {
    {
        cs::Model m = cs::create_model<MakeTake>(Sizes{1, 0, 3, 2}, Sizes{2, 1, 2, 1});
        expect_error([&] { m.setup(); },
                     {"connect('make.m', 'take.pts')", "dimension 1", "the counts must match", "[1,0,3,2]", "[2,1,2,1]"},
                     "same total, other counts");
    }
    {
        cs::Model m = cs::create_model<MakeTake>(Sizes{1, 0, 3, 2}, Sizes{1, 1, 1, 1});
        expect_error([&] { m.setup(); }, {"connect('make.m', 'take.pts')", "the counts must match", "[1,1,1,1]", "[1,0,3,2]"},
                     "another total");
    }
    {
        cs::Model m = cs::create_model<MakeTake>(Sizes{1, 2, 3, 4}, Sizes{1, 2, 3});
        expect_error([&] { m.setup(); },
                     {"connect('make.m', 'take.pts')", "dimension 0", "declares 4", "declares 3", "the extents must match"},
                     "another N");
    }
}

void case_dense_source() {
    cs::Model m = cs::create_model<DenseTop>();
    m.setup();
    m.run();
    m.wait();
    auto sums = m.view_output<DType::f32, 1>("sum.sums");
    sums.sync();
    for (std::size_t i = 0; i < 3; ++i)
        check(sums.span().size() == 3 && sums.span()[i] == static_cast<float>(40 * i + 6), "dense rows: sum");
    auto d = m.view_ragged_output<DType::f32, 2>("gen.d");
    d.sync();
    check(d.n() == 3 && d.block_offsets() == std::vector<std::uint64_t>{0, 4, 8, 12}, "dense rows: offsets");
    check(d.block(2).size() == 4 && d.block(2)[3] == 23.0f, "dense rows: block 2");
    auto in = m.view_ragged_input<DType::f32, 2>("sum.pts");
    in.sync();
    check(flat_of(in) == flat_of(d) && in.block_offsets() == d.block_offsets(), "dense rows: input peer");
    auto dense = m.view_output<DType::f32, 2>("gen.d");
    dense.sync();
    check(dense.span()[5] == 11.0f, "dense rows: the dense view");
}

void case_views() {
    cs::Model m = cs::create_model<Chain>(std::size_t{6});
    m.setup();
    chain_forward(m, {3, 0, 2, 4, 0, 1});
    expect_error([&] { (void)m.view_output<DType::f32, 2>("fill.pts"); }, {"fill.pts", "view_ragged_output"}, "dense view");
    expect_error([&] { (void)m.view_input<DType::f32, 2>("sum.pts"); }, {"sum.pts", "view_ragged_input"}, "dense input view");
    expect_error([&] { (void)m.view_ragged_output<DType::u32, 2>("fill.pts"); }, {"wrong dtype or rank"}, "dtype");
}

void case_errors() {
    {
        cs::Model m = cs::create_model<DenseOnRagged>();
        expect_error([&] { m.setup(); },
                     {"connect('make.m', 'c.in')", "'make.m' is ragged", "a dense Input cannot see per-index extents",
                      "RaggedInput"},
                     "dense input on a ragged source");
    }
    {
        cs::Model m = cs::create_model<HookedOn<FromCounts<DType::i32, 1>>>();
        m.setup();
        m.update_input("c.cnt", cs::init::from_host(std::vector<std::int32_t>{1, -1, 2}));
        expect_error([&] { m.run(); }, {"shape hook on 'c.layout'", "holds a negative value"}, "negative counts");
        m.wait();
        // the model recovers with valid counts
        m.update_input("c.cnt", cs::init::from_host(std::vector<std::int32_t>{1, 1, 2}));
        m.run();
        m.wait();
        auto v = m.view_ragged_output<DType::f32, 2>("c.v");
        v.sync();
        check_ragged(v, blocks_of(std::vector<int>{1, 1, 2}, 100), "after negative counts");
    }
    {
        cs::Model m = cs::create_model<HookedOn<FromCounts<DType::u32, 1>>>();
        m.setup();
        m.update_input("c.cnt", cs::init::from_host(std::vector<std::uint32_t>{4294967295u, 2u}));
        expect_error([&] { m.run(); }, {"shape hook on 'c.layout'", "limited to 2^32 - 1 elements"}, "total past 32 bits");
        m.wait();
    }
    {
        cs::Model m = cs::create_model<HookedOn<FromCounts<DType::u64, 1>>>();
        m.setup();
        m.update_input("c.cnt", cs::init::from_host(std::vector<std::uint64_t>{3, 1ull << 33}));
        expect_error([&] { m.run(); }, {"shape hook on 'c.layout'", "limited to 2^32 - 1 elements"}, "a u64 count past 32 bits");
        m.wait();
    }
}

void case_hooked_output() {
    cs::Model m = cs::create_model<HookedOutTop>();
    m.setup();
    const std::vector<std::vector<std::uint32_t>> runs{
        {1, 2}, {3, 1, 0, 2}, {1, 1, 1, 1, 1, 1, 1, 1, 1}, {2, 0}, {5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5}};
    for (const auto& counts : runs) {
        m.update_input("c.cnt", cs::init::from_host(counts));
        m.run();
        m.wait();
        auto v = m.view_ragged_output<DType::f32, 2>("c.v");
        v.sync();
        check_ragged(v, blocks_of(counts, 100), "hooked output, n = " + std::to_string(counts.size()));
    }
}

void case_fused() {
    Sizes sizes(3000);
    for (std::size_t i = 0; i < sizes.size(); ++i) sizes[i] = (i * 37) % 211;  // zeros and blocks past 64 elements
    cs::Model f = cs::create_model<FusedRagged>(sizes);
    f.setup();
    f.run();
    f.run();
    f.wait();
    cs::Model u = cs::create_model<UnfusedRagged>(sizes);
    u.setup();
    u.run();
    u.wait();
    auto fs = f.view_output<DType::f32, 1>("w.gsum.sums");
    auto is = f.view_output<DType::f32, 1>("w.isum.sums");
    auto us = u.view_output<DType::f32, 1>("gsum.sums");
    fs.sync();
    is.sync();
    us.sync();
    const std::vector<float> a(fs.span().begin(), fs.span().end()), b(us.span().begin(), us.span().end());
    check(a.size() == sizes.size() && a == b, "fused group sums == unfused");
    for (std::size_t i = 0; i < sizes.size() && i < is.span().size(); ++i) {
        float want = 0.0f;
        for (std::size_t j = 0; j < sizes[i]; ++j) want += static_cast<float>(i * 100 + j);
        check(is.span()[i] == want, "fused index-range sums, block " + std::to_string(i));
        if (g_fails) break;
    }
    auto fm = f.view_ragged_output<DType::f32, 2>("w.make.m");
    fm.sync();
    check_ragged(fm, blocks_of(sizes, 100), "fused make.m");
}

int run(const char* name, void (*fn)()) {
    const int before = g_fails;
    try {
        fn();
    } catch (const std::exception& e) {
        std::printf("  FAIL: exception: %s\n", e.what());
        ++g_fails;
    }
    std::printf("%-28s %s\n", name, g_fails == before ? "OK" : "FAIL");
    return g_fails - before;
}

}  // namespace rg

int main() {
    int fails = 0;
    fails += rg::run("chain over forwards", rg::case_chain);
    fails += rg::run("N = 0", rg::case_zero_blocks);
    fails += rg::run("counts_from column 0", rg::case_column0);
    fails += rg::run("offsets_from", rg::case_offsets_from);
    fails += rg::run("declared counts", rg::case_declared_counts);
    fails += rg::run("declared counts mismatch", rg::case_declared_mismatch);
    fails += rg::run("ragged input on dense rows", rg::case_dense_source);
    fails += rg::run("views", rg::case_views);
    fails += rg::run("errors", rg::case_errors);
    fails += rg::run("hooked ragged output", rg::case_hooked_output);
    fails += rg::run("fused group, ragged stages", rg::case_fused);
    std::printf(fails ? "FAILED\n" : "ALL OK\n");
    return fails ? 1 : 0;
}
