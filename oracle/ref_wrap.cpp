// ref_wrap.cpp — TEST INFRASTRUCTURE ONLY: the reference's own plain-C++ oracles behind a C ABI.
//
// Compiled in place against the reference's source tree (REFERENCE_DIR, see oracle/Makefile) into oracle/_ref; no
// reference source is copied into this repository. It exposes:
//   - gemver_chain::make_matrix_A0 / make_vectors / reference_chain / relative_l2
//     (examples/gemver-chain/common/chain_data.hpp:52-161)
//   - nsr::init_cons and nsr::reference_residual<MinMod | VanLeer> (examples/ns-residual/physics.hpp:203-215,
//     reference.hpp:30-130)
// The tests use it to pin the restatement in cspb_oracle.cpp and to generate the golden fixtures under tests/golden.
#include <cstdint>
#include <cstring>
#include <vector>

#include "common/chain_data.hpp"  // examples/gemver-chain
#include "reference.hpp"          // examples/ns-residual (includes physics.hpp)

#define REF_API extern "C" __attribute__((visibility("default")))

REF_API float ref_hash_unit(uint32_t seed, uint64_t index) { return gemver_chain::hash_unit(seed, index); }

REF_API void ref_make_matrix_A0(int64_t n, float* out) {
    const std::vector<float> a = gemver_chain::make_matrix_A0(static_cast<std::size_t>(n));
    std::memcpy(out, a.data(), a.size() * sizeof(float));
}

// the six vectors u1 v1 u2 v2 y z, each n floats, back to back
REF_API void ref_make_vectors(int64_t n, float* out6) {
    const gemver_chain::Vectors v = gemver_chain::make_vectors(static_cast<std::size_t>(n));
    const std::vector<float>* all[] = {&v.u1, &v.v1, &v.u2, &v.v2, &v.y, &v.z};
    for (int k = 0; k < 6; ++k) std::memcpy(out6 + k * n, all[k]->data(), static_cast<std::size_t>(n) * sizeof(float));
}

// reference_chain on the reference's own inputs: out6 = x1 w1 q s x2 w2 (n doubles each); B2 (n*n doubles) if not NULL.
REF_API void ref_reference_chain(int64_t n, double* out6, double* B2) {
    const std::size_t N = static_cast<std::size_t>(n);
    const std::vector<float> A0 = gemver_chain::make_matrix_A0(N);
    const gemver_chain::Vectors g = gemver_chain::make_vectors(N);
    const gemver_chain::ChainResult r = gemver_chain::reference_chain(N, A0, g, B2 != nullptr);
    const std::vector<double>* all[] = {&r.x1, &r.w1, &r.q, &r.s, &r.x2, &r.w2};
    for (int k = 0; k < 6; ++k) std::memcpy(out6 + k * n, all[k]->data(), N * sizeof(double));
    if (B2) std::memcpy(B2, r.B2.data(), N * N * sizeof(double));
}

REF_API double ref_relative_l2(const float* got, const double* want, int64_t n) {
    return gemver_chain::relative_l2(std::vector<float>(got, got + n), std::vector<double>(want, want + n));
}

REF_API void ref_init_cons(int nx, int ny, float amp, float* U) {
    const std::size_t plane = static_cast<std::size_t>(nx) * static_cast<std::size_t>(ny);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            float u[4];
            nsr::init_cons(j, i, amp, u);
            for (int v = 0; v < 4; ++v) U[v * plane + static_cast<std::size_t>(j) * nx + i] = u[v];
        }
}

// reference_residual: R (4, ny, nx) doubles; diag6 = [dt_min, ws_max, sq0..sq3].
REF_API void ref_reference_residual(int nx, int ny, int walls, int limiter, const float* U, double* R, double* diag6) {
    const std::vector<float> u(U, U + 4 * static_cast<std::size_t>(nx) * static_cast<std::size_t>(ny));
    const nsr::RefResult r = limiter == 0 ? nsr::reference_residual<nsr::MinMod>(nx, ny, walls != 0, u)
                                          : nsr::reference_residual<nsr::VanLeer>(nx, ny, walls != 0, u);
    std::memcpy(R, r.R.data(), r.R.size() * sizeof(double));
    diag6[0] = r.dt_min;
    diag6[1] = r.ws_max;
    for (int v = 0; v < 4; ++v) diag6[2 + v] = r.sq[v];
}
