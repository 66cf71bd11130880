// CUDA-graph replay of steady forwards in the cs:: runtime (Model::run), on the GPU (compiled by
// cospanmdao_b200.examples.build_runtime_tests, run by tests/test_examples_gpu.py):
//   - a model of index-range components and a fused group of two work-group stages (a cooperative launch with a grid
//     barrier) is captured once it has run one forward without host waits, and replayed after that;
//   - every forward's results equal the same model run eagerly (NAGA_COSPAN_NO_GRAPH), bit for bit, and a host view
//     made before the forwards shows the last one;
//   - update_input drops the graph: the next forwards use the new values, and a new graph is captured;
//   - a model whose ragged hook reads the device on every forward is never captured.
// Prints one line per case and "ALL OK" when every case passes; exits 1 otherwise.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "naga/cospan/cospan.hpp"

namespace cs = naga::cospan;
using cs::DType;

namespace rp {

int g_fails = 0;
void check(bool ok, const std::string& what) {
    if (!ok) {
        std::printf("  FAIL: %s\n", what.c_str());
        ++g_fails;
    }
}

// z = a x + y
class Axpy : public cs::Component<Axpy> {
public:
    struct Inputs { cs::Input<DType::f32, 1> x, y, a; };
    struct Outputs { cs::Output<DType::f32, 1> z; };
    __host__ __device__ static void compute_forward(sycl::id<1> i, const Inputs& in, const Outputs& out) {
        out.z[i] = in.a[sycl::id<1>{0}] * in.x[i] + in.y[i];
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.x, "x", cs::unspecified);
        declare_input(inputs.y, "y", cs::unspecified);
        declare_input(inputs.a, "a", 1);
        declare_output(outputs.z, "z", cs::unspecified);
    }
    void prepare_forward() override { set_shape(outputs.z, shape_of(inputs.x)[0]); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(outputs.z.shape()));
    }
};

// w[g kWg + l] = v[g kWg + (kWg - 1 - l)] + 1: a work-group stage (reads another work-item's element)
class Reverse : public cs::Component<Reverse> {
public:
    static constexpr std::size_t kWg = 128;
    struct Inputs { cs::Input<DType::f32, 1> v; };
    struct Outputs { cs::Output<DType::f32, 1> w; };
    __host__ __device__ static void compute_forward(cs::GroupItem<1> it, const Inputs& in, const Outputs& out) {
        const std::size_t g = it.get_group(0), l = it.get_local_id(0);
        out.w[sycl::id<1>{g * kWg + l}] = in.v[sycl::id<1>{g * kWg + (kWg - 1 - l)}] + 1.0f;
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.v, "v", cs::unspecified);
        declare_output(outputs.w, "w", cs::unspecified);
    }
    void prepare_forward() override { set_shape(outputs.w, shape_of(inputs.v)[0]); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(inputs.v.shape()), cs::wg_desc(sycl::range<1>{kWg}));
    }
};

class Top : public cs::System {
    std::size_t n_;

public:
    explicit Top(std::size_t n) : n_{n} {}
    void setup() override {
        add_subsystem(cs::subsystem_desc<Axpy>("axpy"));
        add_subsystem(cs::fuse_components("g", cs::connects_desc({{"r1.w", "r2.v"}}), cs::subsystem_desc<Reverse>("r1"),
                                          cs::global_barrier(), cs::subsystem_desc<Reverse>("r2")));
        connect("axpy.z", "g.r1.v");
        init_input("axpy.a", cs::init::fill(1.5f, {1}));
        shape_hook("axpy.x", cs::dim::fixed_at_run(n_));
        shape_hook("axpy.y", cs::dim::fixed_at_run(n_));
    }
};

// a ragged hook: the counts come from the device on every forward
class Counts : public cs::Component<Counts> {
public:
    struct Inputs {
        cs::Input<DType::u32, 1> cnt;
        cs::RaggedInput<DType::f32, 2> layout;
    };
    struct Outputs { cs::RaggedOutput<DType::f32, 2> v; };
    __host__ __device__ static void compute_forward(sycl::id<1> id, const Inputs&, const Outputs& out) {
        auto b = out.v.block(id[0]);
        for (std::size_t j = 0; j < b.size(); ++j) b[j] = static_cast<float>(id[0] + j);
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.cnt, "cnt", cs::unspecified);
        declare_input(inputs.layout, "layout");
        declare_output(outputs.v, "v");
    }
    void prepare_forward() override { set_shape(outputs.v, shape_of(inputs.layout)); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(sycl::range<1>{inputs.layout.size()}));
    }
};
class RaggedTop : public cs::System {
public:
    void setup() override {
        add_subsystem(cs::subsystem_desc<Counts>("c"));
        shape_hook("c.layout", cs::ragged::counts_from("c.cnt"));
    }
};

std::vector<float> values(std::size_t n, float phase) {
    std::vector<float> v(n);
    for (std::size_t i = 0; i < n; ++i) v[i] = static_cast<float>((i * 37) % 101) * 0.25f + phase;
    return v;
}

// the host result of one forward
std::vector<float> expected(const std::vector<float>& x, const std::vector<float>& y) {
    const std::size_t n = x.size(), W = Reverse::kWg;
    std::vector<float> z(n), w1(n), w2(n);
    for (std::size_t i = 0; i < n; ++i) z[i] = 1.5f * x[i] + y[i];
    for (std::size_t i = 0; i < n; ++i) w1[i] = z[(i / W) * W + (W - 1 - i % W)] + 1.0f;
    for (std::size_t i = 0; i < n; ++i) w2[i] = w1[(i / W) * W + (W - 1 - i % W)] + 1.0f;
    return w2;
}

std::vector<float> forwards(bool graphs, std::size_t n, int runs, std::pair<std::uint64_t, std::uint64_t>* counts,
                            std::vector<float>* after_update) {
    if (graphs) unsetenv("NAGA_COSPAN_NO_GRAPH");
    else setenv("NAGA_COSPAN_NO_GRAPH", "1", 1);
    cs::Model m = cs::create_model<Top>(n);
    m.setup();
    m.update_input("axpy.x", cs::init::from_host(values(n, 0.0f)));
    m.update_input("axpy.y", cs::init::from_host(values(n, 3.0f)));
    auto view = m.view_output<DType::f32, 1>("g.r2.w");  // made before the forwards: pushed after each one
    for (int r = 0; r < runs; ++r) m.run();
    m.wait();
    view.sync();
    std::vector<float> out(view.span().begin(), view.span().end());
    // new inputs: the graph is dropped, the forwards use them
    m.update_input("axpy.x", cs::init::from_host(values(n, 7.0f)));
    for (int r = 0; r < runs; ++r) m.run();
    m.wait();
    view.sync();
    if (after_update) after_update->assign(view.span().begin(), view.span().end());
    if (counts) *counts = m.graph_counts();
    return out;
}

void case_replay() {
    const std::size_t n = 128 * 2000;
    std::pair<std::uint64_t, std::uint64_t> cg{}, ce{};
    std::vector<float> g_upd, e_upd;
    const std::vector<float> g = forwards(true, n, 8, &cg, &g_upd);
    const std::vector<float> e = forwards(false, n, 8, &ce, &e_upd);
    unsetenv("NAGA_COSPAN_NO_GRAPH");
    check(g == expected(values(n, 0.0f), values(n, 3.0f)), "graph forwards == host");
    check(g == e, "graph forwards == eager forwards");
    check(g_upd == expected(values(n, 7.0f), values(n, 3.0f)), "after update_input: the new x is used");
    check(g_upd == e_upd, "after update_input: graph == eager");
    // 8 forwards: 1 with the uploads, 1 steady, then a capture and 5 replays; the same again after update_input
    check(cg.first == 2 && cg.second == 10, "captures " + std::to_string(cg.first) + ", replays " + std::to_string(cg.second));
    check(ce.first == 0 && ce.second == 0, "NAGA_COSPAN_NO_GRAPH: no capture");
}

void case_ragged_never_captured() {
    cs::Model m = cs::create_model<RaggedTop>();
    m.setup();
    m.update_input("c.cnt", cs::init::from_host(std::vector<std::uint32_t>{2, 0, 3}));
    for (int r = 0; r < 4; ++r) m.run();
    m.wait();
    check(m.graph_counts().first == 0, "a model with a ragged hook is not captured");
    auto v = m.view_ragged_output<DType::f32, 2>("c.v");
    v.sync();
    check(std::vector<float>(v.span().begin(), v.span().end()) == std::vector<float>{0, 1, 2, 3, 4}, "ragged values");
}

int run(const char* name, void (*fn)()) {
    const int before = g_fails;
    try {
        fn();
    } catch (const std::exception& e) {
        std::printf("  FAIL: exception: %s\n", e.what());
        ++g_fails;
    }
    std::printf("%-32s %s\n", name, g_fails == before ? "OK" : "FAIL");
    return g_fails - before;
}

}  // namespace rp

int main() {
    int fails = 0;
    fails += rp::run("replay of steady forwards", rp::case_replay);
    fails += rp::run("ragged hook: never captured", rp::case_ragged_never_captured);
    std::printf(fails ? "FAILED\n" : "ALL OK\n");
    return fails ? 1 : 0;
}
