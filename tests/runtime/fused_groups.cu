// Fused-group semantics of the cs:: runtime, every case through a cs::Model on the GPU (compiled by
// cospanmdao_b200.examples.build_runtime_tests, run by tests/test_examples_gpu.py). The cases follow the behaviour the
// reference's tests/test_fused_groups.cpp describes: shared local memory carries a stage's values to the next stage of
// the segment, partitioned local memory gives each stage its own slice, an input tie declared by the group reaches
// every member, and a stage with no local memory runs correctly in a launch that has some.
// Prints one line per case and "ALL OK" when every case passes; exits 1 otherwise.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "naga/cospan/cospan.hpp"

namespace cs = naga::cospan;
using cs::DType;

namespace rt {

constexpr std::size_t kWg = 64;
using Tile = cs::LocalMem<cs::LocalArray<DType::f32, 1>>;

// Leave: t[l] = x[g kWg + l] * 2 (shared: the next stage reads it), y = the same
class Leave : public cs::Component<Leave> {
public:
    struct Inputs { cs::Input<DType::f32, 1> x; };
    struct Outputs { cs::Output<DType::f32, 1> y; };
    __host__ __device__ static void compute_forward(cs::GroupItem<1> it, const Inputs& in, const Outputs& out, Tile lm) {
        auto [t] = lm.get(it);
        const std::size_t l = it.get_local_id(0), g = it.get_group(0);
        const float v = in.x[sycl::id<1>{g * kWg + l}] * 2.0f;
        t[l] = v;
        out.y[sycl::id<1>{g * kWg + l}] = v;
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.x, "x", cs::unspecified_shape<1>());
        declare_output(outputs.y, "y", cs::unspecified_shape<1>());
    }
    void prepare_forward() override { set_shape(outputs.y, shape_of(inputs.x)[0]); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(inputs.x.shape()), cs::wg_desc(sycl::range<1>{kWg}),
                                    cs::local_desc(sycl::range<1>{kWg}));
    }
};

// Take: z[g kWg + l] = t[kWg - 1 - l] + scale (after a group barrier: another work-item wrote that element)
class Take : public cs::Component<Take> {
public:
    struct Inputs { cs::Input<DType::f32, 1> x, scale; };
    struct Outputs { cs::Output<DType::f32, 1> z; };
    __host__ __device__ static void compute_forward(cs::GroupItem<1> it, const Inputs& in, const Outputs& out, Tile lm) {
        auto [t] = lm.get(it);
        const std::size_t l = it.get_local_id(0), g = it.get_group(0);
        cs::group_barrier(it.get_group());
        out.z[sycl::id<1>{g * kWg + l}] = t[kWg - 1 - l] + in.scale[sycl::id<1>{0}];
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.x, "x", cs::unspecified_shape<1>());
        declare_input(inputs.scale, "scale", cs::unspecified_shape<1>());
        declare_output(outputs.z, "z", cs::unspecified_shape<1>());
    }
    void prepare_forward() override { set_shape(outputs.z, shape_of(inputs.x)[0]); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(inputs.x.shape()), cs::wg_desc(sycl::range<1>{kWg}),
                                    cs::local_desc(sycl::range<1>{kWg}));
    }
};

// Plain: w[i] = x[i] + 1, a group stage with no local memory
class Plain : public cs::Component<Plain> {
public:
    struct Inputs { cs::Input<DType::f32, 1> x; };
    struct Outputs { cs::Output<DType::f32, 1> w; };
    __host__ __device__ static void compute_forward(cs::GroupItem<1> it, const Inputs& in, const Outputs& out) {
        const std::size_t i = it.get_group(0) * kWg + it.get_local_id(0);
        out.w[sycl::id<1>{i}] = in.x[sycl::id<1>{i}] + 1.0f;
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.x, "x", cs::unspecified_shape<1>());
        declare_output(outputs.w, "w", cs::unspecified_shape<1>());
    }
    void prepare_forward() override { set_shape(outputs.w, shape_of(inputs.x)[0]); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(inputs.x.shape()), cs::wg_desc(sycl::range<1>{kWg}));
    }
};

enum class Case { shared_tile, shared_tile_barrier, partitioned, plain_only, plain_with_local };

class Top : public cs::System {
    Case c_;
    int n_;

public:
    Top(Case c, int n) : c_{c}, n_{n} {}
    void setup() override {
        const auto dn = cs::dim::fixed_at_run(static_cast<std::size_t>(n_));
        switch (c_) {
            case Case::shared_tile:
                // the tie of x is declared by the group; scale is promoted from the group's stage
                add_subsystem(cs::fuse_components(
                    "g", cs::ties_desc({cs::tie_inputs<DType::f32, 1>({"leave.x", "take.x"}, "x")}),
                    cs::segment<cs::local_mem::shared>(cs::subsystem_desc<Leave>("leave"), cs::subsystem_desc<Take>("take"))));
                break;
            case Case::shared_tile_barrier:
                add_subsystem(cs::fuse_components(
                    "g", cs::connects_desc({{"leave.y", "plain.x"}}),
                    cs::ties_desc({cs::tie_inputs<DType::f32, 1>({"leave.x", "take.x"}, "x")}),
                    cs::segment<cs::local_mem::shared>(cs::subsystem_desc<Leave>("leave"), cs::subsystem_desc<Take>("take")),
                    cs::global_barrier(), cs::subsystem_desc<Plain>("plain")));
                break;
            case Case::partitioned:
                add_subsystem(cs::fuse_components(
                    "g", cs::ties_desc({cs::tie_inputs<DType::f32, 1>({"leave.x", "take.x"}, "x")}),
                    cs::segment<cs::local_mem::partitioned>(cs::subsystem_desc<Leave>("leave"), cs::subsystem_desc<Take>("take"))));
                break;
            case Case::plain_only:
                add_subsystem(cs::fuse_components("g", cs::subsystem_desc<Plain>("plain"), cs::global_barrier(),
                                                  cs::subsystem_desc<Plain>("plain2")));
                connect("g.plain.w", "g.plain2.x");
                break;
            case Case::plain_with_local:
                add_subsystem(cs::fuse_components(
                    "g", cs::connects_desc({{"plain.w", "leave.x"}}), cs::subsystem_desc<Plain>("plain"),
                    cs::global_barrier(), cs::subsystem_desc<Leave>("leave")));
                break;
        }
        if (c_ == Case::plain_only || c_ == Case::plain_with_local) {
            shape_hook("g.plain.x", dn);
        } else {
            shape_hook("g.x", dn);
            promote<DType::f32, 1>("g.take.scale", "scale");
            init_input("scale", cs::init::fill(0.5f, {1}));
        }
    }
};

std::vector<float> host_x(int n) {
    std::vector<float> x(static_cast<std::size_t>(n));
    for (int i = 0; i < n; ++i) x[static_cast<std::size_t>(i)] = static_cast<float>((i * 37) % 101) - 50.0f;
    return x;
}

template <int R>
std::vector<float> read(cs::Model& m, const std::string& path) {
    auto v = m.view_output<DType::f32, R>(path);
    v.sync();
    auto s = v.span();
    return std::vector<float>(s.begin(), s.end());
}

int report(const char* name, const std::vector<float>& got, const std::vector<float>& want) {
    std::size_t bad = 0, first = got.size();
    for (std::size_t i = 0; i < want.size(); ++i)
        if (i >= got.size() || got[i] != want[i]) {
            if (first == got.size()) first = i;
            ++bad;
        }
    if (got.size() != want.size() || bad) {
        std::printf("%-24s FAIL: %zu of %zu differ (size %zu)", name, bad, want.size(), got.size());
        if (first < got.size() && first < want.size()) std::printf("; first at %zu: %g, want %g", first, got[first], want[first]);
        std::printf("\n");
        return 1;
    }
    std::printf("%-24s OK\n", name);
    return 0;
}

int run_case(Case c, const char* name, int n) {
    int fails = 0;
    try {
        cs::Model m = cs::create_model<Top>(c, n);
        m.setup();
        const std::vector<float> x = host_x(n);
        const bool plain_in = c == Case::plain_only || c == Case::plain_with_local;
        m.update_input(plain_in ? "g.plain.x" : "g.x", cs::init::from_host(x));
        for (int rep = 0; rep < 2; ++rep) m.run();
        m.wait();
        std::vector<float> y(x.size()), z(x.size()), w(x.size());
        for (std::size_t i = 0; i < x.size(); ++i) {
            y[i] = x[i] * 2.0f;
            w[i] = x[i] + 1.0f;
        }
        for (std::size_t g = 0; g < x.size() / kWg; ++g)
            for (std::size_t l = 0; l < kWg; ++l) z[g * kWg + l] = y[g * kWg + (kWg - 1 - l)] + 0.5f;
        switch (c) {
            case Case::shared_tile:
                fails += report((std::string(name) + " y").c_str(), read<1>(m, "g.leave.y"), y);
                fails += report((std::string(name) + " z").c_str(), read<1>(m, "g.take.z"), z);
                break;
            case Case::shared_tile_barrier: {
                std::vector<float> w2(x.size());
                for (std::size_t i = 0; i < x.size(); ++i) w2[i] = y[i] + 1.0f;
                fails += report((std::string(name) + " z").c_str(), read<1>(m, "g.take.z"), z);
                fails += report((std::string(name) + " w").c_str(), read<1>(m, "g.plain.w"), w2);
                break;
            }
            case Case::partitioned: {
                // partitioned: take reads its own (never written) slice; only leave's output is checked
                fails += report((std::string(name) + " y").c_str(), read<1>(m, "g.leave.y"), y);
                break;
            }
            case Case::plain_only: {
                std::vector<float> w2(x.size());
                for (std::size_t i = 0; i < x.size(); ++i) w2[i] = w[i] + 1.0f;
                fails += report((std::string(name) + " w").c_str(), read<1>(m, "g.plain2.w"), w2);
                break;
            }
            case Case::plain_with_local: {
                std::vector<float> y2(x.size());
                for (std::size_t i = 0; i < x.size(); ++i) y2[i] = w[i] * 2.0f;
                fails += report((std::string(name) + " w").c_str(), read<1>(m, "g.plain.w"), w);
                fails += report((std::string(name) + " y").c_str(), read<1>(m, "g.leave.y"), y2);
                break;
            }
        }
    } catch (const std::exception& e) {
        std::printf("%-24s FAIL: exception: %s\n", name, e.what());
        ++fails;
    }
    return fails;
}

}  // namespace rt

int main() {
    using rt::Case;
    int fails = 0;
    for (int n : {256, 64 * 1000}) {
        std::printf("n = %d\n", n);
        fails += rt::run_case(Case::plain_only, "plain only", n);
        fails += rt::run_case(Case::plain_with_local, "plain + local stage", n);
        fails += rt::run_case(Case::shared_tile, "shared tile", n);
        fails += rt::run_case(Case::shared_tile_barrier, "shared tile + barrier", n);
        fails += rt::run_case(Case::partitioned, "partitioned", n);
    }
    std::printf(fails ? "FAILED\n" : "ALL OK\n");
    return fails ? 1 : 0;
}
