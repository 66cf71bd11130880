// The runtime's fast paths must not replace a component whose arithmetic differs from the reference's (compiled by
// cospanmdao_b200.examples.build_runtime_tests, run by tests/test_examples_gpu.py).
//
// Two GEMVER systems are wired exactly like the reference's Gemver system (Rank2Update -> GemvTPartial ->
// ColReduce<true> -> Gemv, the same port names and the same variables between them), so the runtime recognises both as
// a GEMVER run (patterns.hpp) by type names and wiring. In the first, Gemv computes w = α·Â·x; in the second a
// component also named Gemv computes w = α·Â·x + 1. The first forward runs the components' bodies and the kernel and
// compares them: the honest system then runs cspb_gemver_fused, the decoy keeps its bodies. Both are checked against a
// host f64 evaluation of their OWN arithmetic over two forwards (relative L2 <= 1e-5).
// Prints one line per case and "ALL OK" when every case passes; exits 1 otherwise.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "naga/cospan/cospan.hpp"

namespace cs = naga::cospan;
using cs::DType;

namespace dk {

constexpr std::size_t kR = 64;  // rows per partial-sum strip

// B = A + u1 v1ᵀ + u2 v2ᵀ
class Rank2Update : public cs::Component<Rank2Update> {
public:
    struct Inputs {
        cs::Input<DType::f32, 2> A;
        cs::Input<DType::f32, 1> u1, v1, u2, v2;
    };
    struct Outputs { cs::Output<DType::f32, 2> B; };
    __host__ __device__ static void compute_forward(sycl::id<2> ij, const Inputs& in, const Outputs& out) {
        const sycl::id<1> i{ij[0]}, j{ij[1]};
        out.B[ij] = in.A[ij] + in.u1[i] * in.v1[j] + in.u2[i] * in.v2[j];
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.A, "A", cs::unspecified_shape<2>());
        declare_input(inputs.u1, "u1", cs::unspecified_shape<1>());
        declare_input(inputs.v1, "v1", cs::unspecified_shape<1>());
        declare_input(inputs.u2, "u2", cs::unspecified_shape<1>());
        declare_input(inputs.v2, "v2", cs::unspecified_shape<1>());
        declare_output(outputs.B, "B", cs::unspecified_shape<2>());
    }
    void prepare_forward() override { set_shape(outputs.B, shape_of(inputs.A)[0], shape_of(inputs.A)[1]); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(outputs.B.shape()));
    }
};

// P[c][j] = Σ_{k < kR} B[c·kR + k][j] · y[c·kR + k]
class GemvTPartial : public cs::Component<GemvTPartial> {
public:
    struct Inputs {
        cs::Input<DType::f32, 2> B;
        cs::Input<DType::f32, 1> y;
    };
    struct Outputs { cs::Output<DType::f32, 2> P; };
    __host__ __device__ static void compute_forward(sycl::id<2> cj, const Inputs& in, const Outputs& out) {
        float acc = 0.0f;
        for (std::size_t k = 0; k < kR; ++k) {
            const std::size_t i = cj[0] * kR + k;
            acc += in.B[sycl::id<2>{i, cj[1]}] * in.y[sycl::id<1>{i}];
        }
        out.P[cj] = acc;
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        declare_input(inputs.B, "B", cs::unspecified_shape<2>());
        declare_input(inputs.y, "y", cs::unspecified_shape<1>());
        declare_output(outputs.P, "P", cs::unspecified_shape<2>());
    }
    void prepare_forward() override { set_shape(outputs.P, shape_of(inputs.B)[0] / kR, shape_of(inputs.B)[1]); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return create_launch_config(cs::range_desc(outputs.P.shape()));
    }
};

// x[j] = z[j] + scale · Σ_c P[c][j]
template <bool Z>
class ColReduce : public cs::Component<ColReduce<Z>> {
public:
    struct Inputs {
        cs::Input<DType::f32, 2> P;
        cs::Input<DType::f32, 1> z, scale;
    };
    struct Outputs { cs::Output<DType::f32, 1> x; };
    __host__ __device__ static void compute_forward(sycl::id<1> j, const Inputs& in, const Outputs& out) {
        float acc = 0.0f;
        for (std::size_t c = 0; c < in.P.shape()[0]; ++c) acc += in.P[sycl::id<2>{c, j[0]}];
        out.x[j] = (Z ? in.z[j] : 0.0f) + in.scale[sycl::id<1>{0}] * acc;
    }
    Inputs inputs;
    Outputs outputs;
    void declare() override {
        this->declare_input(inputs.P, "P", cs::unspecified_shape<2>());
        this->declare_input(inputs.z, "z", cs::unspecified_shape<1>());
        this->declare_input(inputs.scale, "scale", cs::unspecified_shape<1>());
        this->declare_output(outputs.x, "x", cs::unspecified_shape<1>());
    }
    void prepare_forward() override { this->set_shape(outputs.x, this->shape_of(inputs.P)[1]); }
    std::unique_ptr<cs::LaunchDescription> define_forward() override {
        return this->create_launch_config(cs::range_desc(outputs.x.shape()));
    }
};

}  // namespace dk

// y[i] = scale · Σ_j B[i][j] x[j] + OFFSET, in a class named Gemv (the runtime knows a component by its unqualified
// type name): the reference's Gemv when OFFSET is 0
#define DK_GEMV(OFFSET)                                                                                             \
    class Gemv : public cs::Component<Gemv> {                                                                       \
    public:                                                                                                         \
        struct Inputs {                                                                                             \
            cs::Input<DType::f32, 2> B;                                                                             \
            cs::Input<DType::f32, 1> x, scale;                                                                      \
        };                                                                                                          \
        struct Outputs { cs::Output<DType::f32, 1> y; };                                                            \
        __host__ __device__ static void compute_forward(sycl::id<1> i, const Inputs& in, const Outputs& out) {      \
            float acc = 0.0f;                                                                                       \
            for (std::size_t j = 0; j < in.B.shape()[1]; ++j) acc += in.B[sycl::id<2>{i[0], j}] * in.x[sycl::id<1>{j}]; \
            out.y[i] = in.scale[sycl::id<1>{0}] * acc + float(OFFSET);                                              \
        }                                                                                                           \
        Inputs inputs;                                                                                              \
        Outputs outputs;                                                                                            \
        void declare() override {                                                                                   \
            declare_input(inputs.B, "B", cs::unspecified_shape<2>());                                               \
            declare_input(inputs.x, "x", cs::unspecified_shape<1>());                                               \
            declare_input(inputs.scale, "scale", cs::unspecified_shape<1>());                                       \
            declare_output(outputs.y, "y", cs::unspecified_shape<1>());                                             \
        }                                                                                                           \
        void prepare_forward() override { set_shape(outputs.y, shape_of(inputs.B)[0]); }                           \
        std::unique_ptr<cs::LaunchDescription> define_forward() override {                                          \
            return create_launch_config(cs::range_desc(outputs.y.shape()));                                         \
        }                                                                                                           \
    };

namespace honest { DK_GEMV(0) }
namespace decoy { DK_GEMV(1) }

template <class G>
class Sys : public cs::System {
    std::size_t n_;

public:
    explicit Sys(std::size_t n) : n_{n} {}
    void setup() override {
        add_subsystem(cs::subsystem_desc<dk::Rank2Update>("r2u"));
        add_subsystem(cs::subsystem_desc<dk::GemvTPartial>("gtp"));
        add_subsystem(cs::subsystem_desc<dk::ColReduce<true>>("cred"));
        add_subsystem(cs::subsystem_desc<G>("gemv"));
        connect("r2u.B", "gtp.B");
        connect("gtp.P", "cred.P");
        connect("r2u.B", "gemv.B");
        connect("cred.x", "gemv.x");
        shape_hook("r2u.A", cs::dim::fixed_at_run(n_), cs::dim::fixed_at_run(n_));
        for (const char* p : {"r2u.u1", "r2u.v1", "r2u.u2", "r2u.v2", "gtp.y", "cred.z"})
            shape_hook(p, cs::dim::fixed_at_run(n_));
        init_input("cred.scale", cs::init::fill(1.2f, {1}));
        init_input("gemv.scale", cs::init::fill(1.5f, {1}));
    }
};

std::vector<float> values(std::size_t n, std::uint32_t seed, float lo, float hi) {
    std::vector<float> v(n);
    std::uint32_t s = seed * 2654435761u + 12345u;
    for (auto& x : v) {
        s = s * 1664525u + 1013904223u;
        x = lo + (hi - lo) * float(s >> 8) * (1.0f / 16777216.0f);
    }
    return v;
}

// w of the f32 inputs in f64, with the component's own offset
std::vector<double> host_w(std::size_t n, const std::vector<std::vector<float>>& in, double offset) {
    const auto &A = in[0], &u1 = in[1], &v1 = in[2], &u2 = in[3], &v2 = in[4], &y = in[5], &z = in[6];
    std::vector<double> B(n * n), x(n, 0.0), w(n, 0.0);
    for (std::size_t i = 0; i < n; ++i)
        for (std::size_t j = 0; j < n; ++j)
            B[i * n + j] = double(A[i * n + j]) + double(u1[i]) * v1[j] + double(u2[i]) * v2[j];
    for (std::size_t i = 0; i < n; ++i)
        for (std::size_t j = 0; j < n; ++j) x[j] += B[i * n + j] * y[i];
    for (std::size_t j = 0; j < n; ++j) x[j] = z[j] + 1.2 * x[j];
    for (std::size_t i = 0; i < n; ++i) {
        double acc = 0.0;
        for (std::size_t j = 0; j < n; ++j) acc += B[i * n + j] * x[j];
        w[i] = 1.5 * acc + offset;
    }
    return w;
}

template <class G>
int run_case(const char* name, double offset) {
    const std::size_t n = 256;
    cs::Model m = cs::create_model<Sys<G>>(n);
    m.setup();
    std::vector<std::vector<float>> in = {values(n * n, 1, -1.f, 1.f), values(n, 2, 0.f, 1.f), values(n, 3, 0.f, 1.f),
                                          values(n, 4, 0.f, 1.f),     values(n, 5, 0.f, 1.f), values(n, 6, 0.f, 1.f),
                                          values(n, 7, 0.f, 1.f)};
    const char* paths[] = {"r2u.A", "r2u.u1", "r2u.v1", "r2u.u2", "r2u.v2", "gtp.y", "cred.z"};
    for (int k = 0; k < 7; ++k) m.update_input(paths[k], cs::init::from_host(in[std::size_t(k)]));
    const std::vector<double> want = host_w(n, in, offset);
    int fails = 0;
    for (int rep = 0; rep < 2; ++rep) {  // the first forward compares kernel and bodies, the second runs the chosen one
        m.run();
        m.wait();
        auto v = m.view_output<DType::f32, 1>("gemv.y");
        v.sync();
        auto s = v.span();
        double num = 0.0, den = 0.0;
        for (std::size_t i = 0; i < n; ++i) {
            num += (double(s[i]) - want[i]) * (double(s[i]) - want[i]);
            den += want[i] * want[i];
        }
        const double rel = std::sqrt(num / den);
        const bool ok = rel <= 1e-5;
        std::printf("%-8s forward %d: w relative L2 %.3g against its own arithmetic %s\n", name, rep, rel,
                    ok ? "OK" : "FAIL");
        fails += ok ? 0 : 1;
    }
    return fails;
}

int main() {
    int fails = 0;
    try {
        fails += run_case<honest::Gemv>("honest", 0.0);
        fails += run_case<decoy::Gemv>("decoy", 1.0);
    } catch (const std::exception& e) {
        std::printf("exception: %s\n", e.what());
        fails += 1;
    }
    std::printf(fails ? "FAILED\n" : "ALL OK\n");
    return fails ? 1 : 0;
}
