// cspb_oracle.cpp — TEST INFRASTRUCTURE ONLY: the CPU oracle of the cspb kernels.
//
// A restatement, in plain C++ (f64 unless noted), of what the reference computes on the hot path. Only the tests, the
// smoke check and the benchmark's CPU-baseline leg load it, as a checker and a timed baseline; the product path
// (libcspb.so and the host runtime) never calls it. Built with -ffp-contract=off so that every f32 restatement rounds
// exactly where the source says. Each function names the reference code it follows; the reference's own plain-C++
// oracles (gemver_chain::reference_chain, nsr::reference_residual) are compiled separately in place (ref_wrap.cpp,
// oracle/_ref) and the tests pin this restatement against them.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_API extern "C" __attribute__((visibility("default")))

namespace {

// ---- the seeded generator: gemver_chain::mix32 / hash_unit (examples/gemver-chain/common/chain_data.hpp:34-49) ----
inline uint32_t mix(uint32_t x) {
    x = (x ^ (x >> 16)) * 0x7feb352du;
    x = (x ^ (x >> 15)) * 0x846ca68bu;
    return x ^ (x >> 16);
}
inline uint32_t hash24(uint32_t seed, uint64_t i) {
    const uint32_t a = mix(seed * 0x9e3779b9u + 0x85ebca6bu);
    const uint32_t b = mix(static_cast<uint32_t>(i) + mix(static_cast<uint32_t>(i >> 32) + seed));
    return mix(a ^ b) >> 8;
}

}  // namespace

// ==================================================================================================================
// Generators
// ==================================================================================================================

// dist 0: hash_unit in [-1, 1); dist 1: h · 2^-24 in [0, 1).
ORC_API void orc_fill_hash(float* out, int64_t count, uint64_t base, uint32_t seed, int dist) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < count; ++i) {
        const uint32_t h = hash24(seed, base + static_cast<uint64_t>(i));
        out[i] = dist == 0 ? static_cast<float>(h) * (1.0f / 8388608.0f) - 1.0f : static_cast<float>(h) * (1.0f / 16777216.0f);
    }
}

// ==================================================================================================================
// GEMVER family, f64 (the gemver lambda and the BiCGK loop of reference_chain, chain_data.hpp:93-144, generalized to
// independent α, β and a z that may be absent). B(i, j) = A(i, j) + u1[i]·v1[j] + u2[i]·v2[j] is formed in f64 from the
// f32 operands on the fly (O(n) memory), exactly as the reference's oracle does.
// ==================================================================================================================

namespace {
struct Gv {
    int64_t n, lda;
    const float* A;
    const float *u1, *v1, *u2, *v2;
    double b(int64_t i, int64_t j) const {
        return static_cast<double>(A[i * lda + j]) + (static_cast<double>(u1[i]) * v1[j] + static_cast<double>(u2[i]) * v2[j]);
    }
};

// acc[j] = Σ_i B(i, j) · y[i], in blocks of rows with per-thread accumulators combined in a fixed order.
void colsum64(const Gv& g, const double* y, double* acc) {
    const int64_t n = g.n;
    std::fill(acc, acc + n, 0.0);
#pragma omp parallel
    {
        std::vector<double> loc(static_cast<size_t>(n), 0.0);
#pragma omp for schedule(static) nowait
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = 0; j < n; ++j) loc[j] += g.b(i, j) * y[i];
#pragma omp critical
        for (int64_t j = 0; j < n; ++j) acc[j] += loc[j];
    }
}
void rowdot64(const Gv& g, const double* x, double* out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < g.n; ++i) {
        double s = 0.0;
        for (int64_t j = 0; j < g.n; ++j) s += g.b(i, j) * x[j];
        out[i] = s;
    }
}
}  // namespace

// x = β·Bᵀy + z (z may be NULL), w = α·B·x; B_out (f64, optional) receives B.
ORC_API void orc_gemver_f64(int64_t n, int64_t lda, const float* A, const float* u1, const float* v1, const float* u2,
                            const float* v2, const float* y, const float* z, double alpha, double beta, double* x,
                            double* w, double* B_out) {
    const Gv g{n, lda, A, u1, v1, u2, v2};
    std::vector<double> yd(y, y + n), acc(static_cast<size_t>(n));
    colsum64(g, yd.data(), acc.data());
    for (int64_t j = 0; j < n; ++j) x[j] = (z ? static_cast<double>(z[j]) : 0.0) + beta * acc[j];
    rowdot64(g, x, acc.data());
    for (int64_t i = 0; i < n; ++i) w[i] = alpha * acc[i];
    if (B_out) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = 0; j < n; ++j) B_out[i * n + j] = g.b(i, j);
    }
}

// q = B·p, s = Bᵀ·r with B given in f32 (lda row stride).
ORC_API void orc_bicgk_f64(int64_t n, int64_t ldb, const float* B, const float* p, const float* r, double* q, double* s) {
    static const float zero = 0.0f;
    std::vector<float> zv(static_cast<size_t>(n), zero);
    const Gv g{n, ldb, B, zv.data(), zv.data(), zv.data(), zv.data()};
    std::vector<double> pd(p, p + n), rd(r, r + n);
    rowdot64(g, pd.data(), q);
    colsum64(g, rd.data(), s);
}

// The chain G1 -> BiCGK -> G2 of reference_chain (chain_data.hpp:93-144) with general α, β and separate G2 vectors:
// B1 = A0 + U_a, B2 = B1 + U_b with U = u1·v1ᵀ + u2·v2ᵀ, all formed in f64.
ORC_API void orc_chain_f64(int64_t n, const float* A0, const float* u1a, const float* v1a, const float* u2a,
                           const float* v2a, const float* ya, const float* za, const float* u1b, const float* v1b,
                           const float* u2b, const float* v2b, double alpha, double beta, double* x1, double* w1,
                           double* q, double* s, double* x2, double* w2, double* B2_out) {
    auto b1 = [&](int64_t i, int64_t j) {
        return static_cast<double>(A0[i * n + j]) +
               (static_cast<double>(u1a[i]) * v1a[j] + static_cast<double>(u2a[i]) * v2a[j]);
    };
    auto b2 = [&](int64_t i, int64_t j) {
        return b1(i, j) + (static_cast<double>(u1b[i]) * v1b[j] + static_cast<double>(u2b[i]) * v2b[j]);
    };
    std::vector<double> acc(static_cast<size_t>(n));
    auto colsum = [&](auto&& bij, const double* y, double* out) {
        std::fill(out, out + n, 0.0);
#pragma omp parallel
        {
            std::vector<double> loc(static_cast<size_t>(n), 0.0);
#pragma omp for schedule(static) nowait
            for (int64_t i = 0; i < n; ++i)
                for (int64_t j = 0; j < n; ++j) loc[j] += bij(i, j) * y[i];
#pragma omp critical
            for (int64_t j = 0; j < n; ++j) out[j] += loc[j];
        }
    };
    auto rowdot = [&](auto&& bij, const double* x, double* out) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            double t = 0.0;
            for (int64_t j = 0; j < n; ++j) t += bij(i, j) * x[j];
            out[i] = t;
        }
    };
    std::vector<double> yd(ya, ya + n);
    colsum(b1, yd.data(), acc.data());
    for (int64_t j = 0; j < n; ++j) x1[j] = (za ? static_cast<double>(za[j]) : 0.0) + beta * acc[j];
    rowdot(b1, x1, q);
    for (int64_t i = 0; i < n; ++i) w1[i] = alpha * q[i];
    colsum(b1, w1, s);
    colsum(b2, q, acc.data());
    for (int64_t j = 0; j < n; ++j) x2[j] = s[j] + beta * acc[j];
    rowdot(b2, x2, acc.data());
    for (int64_t i = 0; i < n; ++i) w2[i] = alpha * acc[i];
    if (B2_out) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = 0; j < n; ++j) B2_out[i * n + j] = b2(i, j);
    }
}

// ==================================================================================================================
// GEMVER in f32, the order of the reference's UNFUSED components (examples/gemver-chain/components.hpp):
//   Rank2Update  B[i][j] = (A + u1[i]·v1[j]) + u2[i]·v2[j]                 (:85-97)
//   GemvTPartial P[c][j] = Σ_{k<R} B[cR+k][j]·y[cR+k], k ascending          (:142-167)
//   ColReduce    x[j] = z[j] + β·Σ_c P[c][j], c ascending                    (:192-219)
//   Gemv         w[i] = α·Σ_j B[i][j]·x[j]; per work-item l the terms j ≡ l (mod 256) ascending, then the 256 partial
//                sums combined by a binary tree (reduce_over_group's order is the implementation's; a tree is used)
// OpenMP over strips / rows. The timed CPU baseline of the GEMVER benchmark, and a tolerance check of the kernels.
// B may be NULL (only the matrix-free quantities are wanted): B is then recomputed where it is read.
// ==================================================================================================================
ORC_API void orc_gemver_f32_unfused(int64_t n, int64_t R, const float* A, const float* u1, const float* v1,
                                    const float* u2, const float* v2, const float* y, const float* z, float alpha,
                                    float beta, float* B, float* x, float* w, int64_t row_begin, int64_t row_end) {
    // row_begin / row_end bound the rows processed (a bounded sample for timing); the full GEMVER uses 0, n.
    const int64_t strips_lo = row_begin / R, strips_hi = (row_end + R - 1) / R;
    const int64_t strips = n / R;
    std::vector<float> P(static_cast<size_t>(std::max<int64_t>(strips, 1)) * static_cast<size_t>(n), 0.0f);
    auto bij = [&](int64_t i, int64_t j) {
        const float t = A[i * n + j] + u1[i] * v1[j];
        return t + u2[i] * v2[j];
    };
#pragma omp parallel for schedule(static)
    for (int64_t c = strips_lo; c < strips_hi; ++c) {
        float* Pc = P.data() + c * n;
        for (int64_t j = 0; j < n; ++j) Pc[j] = 0.0f;
        for (int64_t k = 0; k < R; ++k) {
            const int64_t i = c * R + k;
            const float yi = y[i];
            for (int64_t j = 0; j < n; ++j) {
                const float b = bij(i, j);
                if (B) B[i * n + j] = b;
                Pc[j] += b * yi;
            }
        }
    }
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < n; ++j) {
        float acc = 0.0f;
        for (int64_t c = strips_lo; c < strips_hi; ++c) acc += P[c * n + j];
        x[j] = (z ? z[j] : 0.0f) + beta * acc;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = row_begin; i < row_end; ++i) {
        float part[256];
        for (int l = 0; l < 256; ++l) {
            float acc = 0.0f;
            for (int64_t j = l; j < n; j += 256) acc += (B ? B[i * n + j] : bij(i, j)) * x[j];
            part[l] = acc;
        }
        for (int width = 128; width >= 1; width >>= 1)
            for (int l = 0; l < width; ++l) part[l] = part[l] + part[l + width];
        w[i] = alpha * part[0];
    }
}

// ==================================================================================================================
// Compressible NS residual (examples/ns-residual): physics.hpp restated, reference_residual (reference.hpp:30-130)
// restated. Templated on the scalar: f64 is the oracle; f32 with the reference's tile arithmetic is the timed CPU
// baseline. Conventions (physics.hpp:14-31): arrays (4, ny, nx) row-major; primitives (ρ, u, v, p); x periodic, y
// periodic or no-slip adiabatic walls (ghost = mirror with both momenta negated); MUSCL on primitives with a
// limiter, HLLC with Davis speeds, viscous flux from face-normal differences and averaged cell gradients.
// ==================================================================================================================
namespace nsc {

constexpr double kG = 1.4, kMu = 0.01, kPr = 0.72, kCfl = 0.5;

template <class T> inline T mn(T a, T b) { return a < b ? a : b; }
template <class T> inline T mx(T a, T b) { return a > b ? a : b; }

// limiters of physics.hpp:62-80: zero at an extremum
template <class T> inline T slope(int lim, T a, T b) {
    if (lim == 0) {
        if (a * b <= T(0)) return T(0);
        return a > T(0) ? mn(a, b) : mx(a, b);
    }
    const T ab = a * b;
    if (ab <= T(0)) return T(0);
    return T(2) * ab / (a + b);
}

template <class T> inline void cons_to_prim(const T* U, T* W) {  // physics.hpp:86-94
    const T rho = U[0], u = U[1] / rho, v = U[2] / rho;
    W[0] = rho;
    W[1] = u;
    W[2] = v;
    W[3] = (T(kG) - T(1)) * (U[3] - T(0.5) * rho * (u * u + v * v));
}

// (ux, uy, vx, vy, Tx, Ty) by central differences of the four neighbours (physics.hpp:97-104), T = p/ρ
template <class T> inline void cell_grad(const T* w_w, const T* w_e, const T* w_s, const T* w_n, T* g) {
    g[0] = T(0.5) * (w_e[1] - w_w[1]);
    g[1] = T(0.5) * (w_n[1] - w_s[1]);
    g[2] = T(0.5) * (w_e[2] - w_w[2]);
    g[3] = T(0.5) * (w_n[2] - w_s[2]);
    g[4] = T(0.5) * (w_e[3] / w_e[0] - w_w[3] / w_w[0]);
    g[5] = T(0.5) * (w_n[3] / w_n[0] - w_s[3] / w_s[0]);
}

// HLLC through a face normal to x (d = 0) or y (d = 1), physics.hpp:109-152 (Toro's HLLC, Davis speeds)
template <class T> inline void flux_hllc(const T* L, const T* R, int d, T* F) {
    const T g = T(kG);
    const int n = d == 0 ? 1 : 2, t = d == 0 ? 2 : 1;
    const T rl = L[0], rr = R[0], pl = L[3], pr = R[3];
    const T ul = L[n], vl = L[t], ur = R[n], vr = R[t];
    const T cl = std::sqrt(g * pl / rl), cr = std::sqrt(g * pr / rr);
    const T El = pl / (g - T(1)) + T(0.5) * rl * (ul * ul + vl * vl);
    const T Er = pr / (g - T(1)) + T(0.5) * rr * (ur * ur + vr * vr);
    const T sl = mn(ul - cl, ur - cr), sr = mx(ul + cl, ur + cr);
    const T sm = (pr - pl + rl * ul * (sl - ul) - rr * ur * (sr - ur)) / (rl * (sl - ul) - rr * (sr - ur));
    T f[4];
    auto side = [&](T r, T un, T ut, T p, T E) {
        f[0] = r * un;
        f[1] = r * un * un + p;
        f[2] = r * un * ut;
        f[3] = (E + p) * un;
    };
    auto star = [&](T r, T un, T ut, T p, T E, T s) {
        const T k = r * (s - un) / (s - sm);
        const T Es = k * (E / r + (sm - un) * (sm + p / (r * (s - un))));
        f[0] = r * un + s * (k - r);
        f[1] = r * un * un + p + s * (k * sm - r * un);
        f[2] = r * un * ut + s * (k * ut - r * ut);
        f[3] = (E + p) * un + s * (Es - E);
    };
    if (sl >= T(0)) side(rl, ul, vl, pl, El);
    else if (sr <= T(0)) side(rr, ur, vr, pr, Er);
    else if (sm >= T(0)) star(rl, ul, vl, pl, El, sl);
    else star(rr, ur, vr, pr, Er, sr);
    F[0] = f[0];
    F[n] = f[1];
    F[t] = f[2];
    F[3] = f[3];
}

// Newtonian viscous flux with Fourier heat flux (physics.hpp:157-192)
template <class T> inline void flux_visc(const T* L, const T* R, const T* gl, const T* gr, int d, T* F) {
    const T uf = T(0.5) * (L[1] + R[1]), vf = T(0.5) * (L[2] + R[2]);
    const T TL = L[3] / L[0], TR = R[3] / R[0];
    T ux, uy, vx, vy, Tx, Ty;
    if (d == 0) {
        ux = R[1] - L[1];
        vx = R[2] - L[2];
        Tx = TR - TL;
        uy = T(0.5) * (gl[1] + gr[1]);
        vy = T(0.5) * (gl[3] + gr[3]);
        Ty = T(0.5) * (gl[5] + gr[5]);
    } else {
        uy = R[1] - L[1];
        vy = R[2] - L[2];
        Ty = TR - TL;
        ux = T(0.5) * (gl[0] + gr[0]);
        vx = T(0.5) * (gl[2] + gr[2]);
        Tx = T(0.5) * (gl[4] + gr[4]);
    }
    const T mu = T(kMu), kt = mu * T(kG) / ((T(kG) - T(1)) * T(kPr));
    const T dv = ux + vy;
    const T sxx = mu * (T(2) * ux - T(2) / T(3) * dv);
    const T syy = mu * (T(2) * vy - T(2) / T(3) * dv);
    const T sxy = mu * (uy + vx);
    F[0] = T(0);
    if (d == 0) {
        F[1] = sxx;
        F[2] = sxy;
        F[3] = uf * sxx + vf * sxy + kt * Tx;
    } else {
        F[1] = sxy;
        F[2] = syy;
        F[3] = uf * sxy + vf * syy + kt * Ty;
    }
}

// local time step and wave speed (physics.hpp:196-202)
template <class T> inline void diag(const T* W, T& dt, T& ws) {
    const T c = std::sqrt(T(kG) * W[3] / W[0]);
    const T ax = (W[1] < T(0) ? -W[1] : W[1]) + c, ay = (W[2] < T(0) ? -W[2] : W[2]) + c;
    const T nu = T(kMu) / W[0] * mx(T(4) / T(3), T(kG) / T(kPr));
    dt = T(kCfl) / (ax + ay + T(4) * nu);
    ws = mx(ax, ay);
}

inline long wrapl(long k, long n) { return ((k % n) + n) % n; }

// The residual of every cell. Primitives of the domain padded by 2 (ghost cells by the boundary rule), then, per cell,
// R = -((Fc_e - Fc_w) + (Fc_n - Fc_s)) + ((Fv_e - Fv_w) + (Fv_n - Fv_s)) with each face flux evaluated once from the
// two cells beside it.
template <class T>
void residual(int nx, int ny, bool walls, int lim, const float* U, T* Rout, double* dt_min, double* ws_max, double* sq) {
    const long PX = nx + 4, PY = ny + 4;
    std::vector<T> W(static_cast<size_t>(4 * PX * PY));
    auto wp = [&](int c, long b, long a) -> T& { return W[static_cast<size_t>((c * PY + b) * PX + a)]; };
#pragma omp parallel for schedule(static)
    for (long b = 0; b < PY; ++b)
        for (long a = 0; a < PX; ++a) {
            const long j = b - 2, i = a - 2, is = wrapl(i, nx);
            long js = j;
            T sgn = T(1);
            if (j < 0 || j >= ny) {
                if (walls) {
                    js = j < 0 ? -1 - j : 2L * ny - 1 - j;
                    sgn = T(-1);
                } else {
                    js = wrapl(j, ny);
                }
            }
            T c[4], w[4];
            for (int v = 0; v < 4; ++v) c[v] = static_cast<T>(U[(static_cast<long>(v) * ny + js) * nx + is]);
            c[1] = c[1] * sgn;
            c[2] = c[2] * sgn;
            cons_to_prim<T>(c, w);
            for (int v = 0; v < 4; ++v) wp(v, b, a) = w[v];
        }
    auto prim = [&](long b, long a, T* w) { for (int v = 0; v < 4; ++v) w[v] = wp(v, b, a); };
    auto slopes = [&](long b, long a, int d, T* s) {
        for (int v = 0; v < 4; ++v) {
            const T w0 = wp(v, b, a);
            const T wm = d == 0 ? wp(v, b, a - 1) : wp(v, b - 1, a);
            const T wq = d == 0 ? wp(v, b, a + 1) : wp(v, b + 1, a);
            s[v] = slope<T>(lim, w0 - wm, wq - w0);
        }
    };
    auto grad = [&](long b, long a, T* g) {
        T w_w[4], w_e[4], w_s[4], w_n[4];
        prim(b, a - 1, w_w);
        prim(b, a + 1, w_e);
        prim(b - 1, a, w_s);
        prim(b + 1, a, w_n);
        cell_grad<T>(w_w, w_e, w_s, w_n, g);
    };
    // the face between cell (bl, al) and its east (d = 0) or north (d = 1) neighbour
    auto face = [&](long bl, long al, int d, T* Fc, T* Fv) {
        const long br = d == 0 ? bl : bl + 1, ar = d == 0 ? al + 1 : al;
        T pl[4], pr[4], sl[4], sr[4], wl[4], wr[4], gl[6], gr[6];
        prim(bl, al, pl);
        prim(br, ar, pr);
        slopes(bl, al, d, sl);
        slopes(br, ar, d, sr);
        for (int v = 0; v < 4; ++v) {
            wl[v] = pl[v] + T(0.5) * sl[v];
            wr[v] = pr[v] - T(0.5) * sr[v];
        }
        flux_hllc<T>(wl, wr, d, Fc);
        grad(bl, al, gl);
        grad(br, ar, gr);
        flux_visc<T>(pl, pr, gl, gr, d, Fv);
    };
    // Faces once each: per thread, row buffers of the x-faces of a row and the y-faces below / above it (the thread's
    // first row computes its lower y-faces; later rows reuse the previous row's upper ones).
    double dmin = 1e300, wmax = -1e300, s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma omp parallel reduction(min : dmin) reduction(max : wmax) reduction(+ : s0, s1, s2, s3)
    {
        std::vector<T> fcx(4 * static_cast<size_t>(nx + 1)), fvx(fcx.size());
        std::vector<T> fcy0(4 * static_cast<size_t>(nx)), fvy0(fcy0.size()), fcy1(fcy0.size()), fvy1(fcy0.size());
        long prev = -2;
#pragma omp for schedule(static)
        for (long j = 0; j < ny; ++j) {
            const long b = j + 2;
            if (j != prev + 1)
                for (long i = 0; i < nx; ++i) face(b - 1, i + 2, 1, &fcy1[4 * i], &fvy1[4 * i]);
            prev = j;
            std::swap(fcy0, fcy1);
            std::swap(fvy0, fvy1);
            for (long i = 0; i < nx; ++i) face(b, i + 2, 1, &fcy1[4 * i], &fvy1[4 * i]);
            for (long i = 0; i <= nx; ++i) face(b, i + 1, 0, &fcx[4 * i], &fvx[4 * i]);
            for (long i = 0; i < nx; ++i) {
                T w[4];
                prim(b, i + 2, w);
                T dt, ws;
                diag<T>(w, dt, ws);
                dmin = std::min(dmin, static_cast<double>(dt));
                wmax = std::max(wmax, static_cast<double>(ws));
                double sqv[4];
                for (int v = 0; v < 4; ++v) {
                    const size_t x0 = 4 * static_cast<size_t>(i) + v, x1 = x0 + 4;
                    const T divc = (fcx[x1] - fcx[x0]) + (fcy1[x0] - fcy0[x0]);
                    const T divv = (fvx[x1] - fvx[x0]) + (fvy1[x0] - fvy0[x0]);
                    const T r = -divc + divv;
                    Rout[(static_cast<long>(v) * ny + j) * nx + i] = r;
                    sqv[v] = static_cast<double>(r) * static_cast<double>(r);
                }
                s0 += sqv[0];
                s1 += sqv[1];
                s2 += sqv[2];
                s3 += sqv[3];
            }
        }
    }
    if (dt_min) *dt_min = dmin;
    if (ws_max) *ws_max = wmax;
    if (sq) { sq[0] = s0; sq[1] = s1; sq[2] = s2; sq[3] = s3; }
}

}  // namespace nsc

// f64 oracle. R (4, ny, nx) doubles; diag[6] = [dt_min, ws_max, sq0..3].
ORC_API void orc_ns_comp_f64(int nx, int ny, int walls, int limiter, const float* U, double* R, double* diag6) {
    nsc::residual<double>(nx, ny, walls != 0, limiter, U, R, diag6, diag6 + 1, diag6 + 2);
}
// f32 restatement (the timed CPU baseline).
ORC_API void orc_ns_comp_f32(int nx, int ny, int walls, int limiter, const float* U, float* R, double* diag6) {
    nsc::residual<float>(nx, ny, walls != 0, limiter, U, R, diag6, diag6 + 1, diag6 + 2);
}

// The initial field (physics.hpp:203-215) in f32 with libm's sinf / cosf.
ORC_API void orc_ns_init_cons(int nx, int ny, float amp, float* U) {
    const float k = static_cast<float>(2.0 * 3.14159265358979323846 / 32.0);
    const size_t plane = static_cast<size_t>(nx) * ny;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const float x = static_cast<float>(i) + 0.5f, y = static_cast<float>(j) + 0.5f;
            const float sx = std::sin(k * x), cx = std::cos(k * x), sy = std::sin(k * y), cy = std::cos(k * y);
            const float r = 1.0f + 0.1f * amp * sx * sy;
            const float u = 0.3f + 0.05f * amp * cx * sy;
            const float v = 0.2f + 0.05f * amp * sx * cy;
            const float p = 1.0f + 0.05f * amp * cx * cy;
            const size_t c = static_cast<size_t>(j) * nx + i;
            U[c] = r;
            U[plane + c] = r * u;
            U[2 * plane + c] = r * v;
            U[3 * plane + c] = p / (static_cast<float>(nsc::kG) - 1.0f) + 0.5f * r * (u * u + v * v);
        }
}

// ==================================================================================================================
// Incompressible NS residual (the workload's formula; no reference code computes it). f64 from f32 fields, periodic.
// norms[3] = ||r_u||, ||r_v||, ||r_c||. R outputs may be NULL.
// ==================================================================================================================
ORC_API void orc_ns_incomp_f64(int nx, int ny, double h, double nu, const float* u, const float* v, const float* p,
                               double* ru, double* rv, double* rc, double* norms) {
    const double i2h = 1.0 / (2.0 * h), ih2 = 1.0 / (h * h);
    double su = 0, sv = 0, sc = 0;
#pragma omp parallel for schedule(static) reduction(+ : su, sv, sc)
    for (int j = 0; j < ny; ++j) {
        const int jn = (j + 1) % ny, js = (j + ny - 1) % ny;
        for (int i = 0; i < nx; ++i) {
            const int ie = (i + 1) % nx, iw = (i + nx - 1) % nx;
            auto at = [&](const float* f, int jj, int ii) { return static_cast<double>(f[static_cast<size_t>(jj) * nx + ii]); };
            const double uc = at(u, j, i), vc = at(v, j, i);
            const double uE = at(u, j, ie), uW = at(u, j, iw), uN = at(u, jn, i), uS = at(u, js, i);
            const double vE = at(v, j, ie), vW = at(v, j, iw), vN = at(v, jn, i), vS = at(v, js, i);
            const double pE = at(p, j, ie), pW = at(p, j, iw), pN = at(p, jn, i), pS = at(p, js, i);
            const double dudx = (uE - uW) * i2h, dudy = (uN - uS) * i2h;
            const double dvdx = (vE - vW) * i2h, dvdy = (vN - vS) * i2h;
            const double dpdx = (pE - pW) * i2h, dpdy = (pN - pS) * i2h;
            const double lu = (((uE - uc) + (uW - uc)) + ((uN - uc) + (uS - uc))) * ih2;
            const double lv = (((vE - vc) + (vW - vc)) + ((vN - vc) + (vS - vc))) * ih2;
            const double a = uc * dudx + vc * dudy + dpdx - nu * lu;
            const double b = uc * dvdx + vc * dvdy + dpdy - nu * lv;
            const double c = dudx + dvdy;
            const size_t k = static_cast<size_t>(j) * nx + i;
            if (ru) ru[k] = a;
            if (rv) rv[k] = b;
            if (rc) rc[k] = c;
            su += a * a;
            sv += b * b;
            sc += c * c;
        }
    }
    if (norms) {
        norms[0] = std::sqrt(su);
        norms[1] = std::sqrt(sv);
        norms[2] = std::sqrt(sc);
    }
}

// ==================================================================================================================
// Scans (std::exclusive_scan + total, tests/test_device_scan.cpp:48-53) and the ragged column (build_column,
// cospanmdao/include/naga/cospan/shape_hook.hpp:215-348).
// ==================================================================================================================
ORC_API void orc_exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n) {
    uint32_t run = 0;
    for (int64_t i = 0; i < n; ++i) {
        out[i] = run;
        run += in[i];
    }
    out[n] = run;
}
ORC_API void orc_exclusive_scan_u64(const uint64_t* in, uint64_t* out, int64_t n) {
    uint64_t run = 0;
    for (int64_t i = 0; i < n; ++i) {
        out[i] = run;
        run += in[i];
    }
    out[n] = run;
}

// dtype: 0 i32, 1 u32, 2 i64, 3 u64. total_flag[2] = [offs[N], flag].
ORC_API void orc_build_column(const void* src, int dtype, int64_t count, int64_t k, int offsets_mode, uint32_t* extents,
                              uint32_t* offs, uint32_t* total_flag) {
    uint32_t flag = 0;
    auto narrow = [&](int64_t idx, bool& neg) -> uint32_t {
        neg = false;
        switch (dtype) {
            case 0: { const int32_t v = static_cast<const int32_t*>(src)[idx]; if (v < 0) { neg = true; return 0; } return static_cast<uint32_t>(v); }
            case 1: return static_cast<const uint32_t*>(src)[idx];
            case 2: {
                const int64_t v = static_cast<const int64_t*>(src)[idx];
                if (v < 0) { neg = true; return 0; }
                if (v > 0xffffffffLL) { flag |= 2u; return 0; }
                return static_cast<uint32_t>(v);
            }
            default: {
                const uint64_t v = static_cast<const uint64_t*>(src)[idx];
                if (v > 0xffffffffULL) { flag |= 2u; return 0; }
                return static_cast<uint32_t>(v);
            }
        }
    };
    if (!offsets_mode) {
        const int64_t n = count;
        uint64_t run = 0;
        for (int64_t i = 0; i < n; ++i) {
            bool neg;
            const uint32_t x = narrow(i * k, neg);
            if (neg) flag |= 1u;
            extents[i] = x;
            offs[i] = static_cast<uint32_t>(run);
            run += x;
        }
        offs[n] = static_cast<uint32_t>(run);
        if (run > 0xffffffffULL) flag |= 2u;
    } else {
        const int64_t n = count - 1;
        for (int64_t i = 0; i < count; ++i) {
            bool neg;
            const uint32_t x = narrow(i, neg);
            if (neg || (i == 0 && x != 0)) flag |= 1u;
            offs[i] = x;
        }
        for (int64_t i = 0; i < n; ++i) {
            if (offs[i + 1] < offs[i]) {
                extents[i] = 0;
                flag |= 1u;
            } else {
                extents[i] = offs[i + 1] - offs[i];
            }
        }
    }
    total_flag[0] = offs[offsets_mode ? count - 1 : count];
    total_flag[1] = flag;
}

ORC_API int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
