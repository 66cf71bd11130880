// naga/cospan/patterns.hpp — leaves that run as one cspb kernel instead of their own component bodies.
//
// At finalize, the runtime looks through its leaves (solo components and fused groups, in run order) for runs of
// components that together compute something a cspb kernel computes in fewer passes over memory, and registers a fast
// path for them: the first leaf of the run calls the kernel through the C ABI (include/cspb.h), the others are
// skipped. Everything else still runs its own bodies. A run is recognised by its component types and by its wiring
// (which ports share a variable), never by names or paths, so every style that the reference's gemver-chain example
// builds (unfused, parallel, fused, naive, onepass, crafted) lands on the same kernel:
//
//   GEMVER   Rank2Update | Rank2UpdateLocal → GemvTPartial | GemvTPartialLocal → ColReduce<true> → Gemv
//            (examples/gemver-chain/components.hpp:85-265, :366-470)             → cspb_gemver_fused
//   BiCGK    BicgkOnePass → RowReduce → ColReduce<false>   (components.hpp:277-358) → cspb_bicgk_fused
//            Gemv → GemvTPartial → ColReduce<false>        (the unfused / parallel / fused BiCGK)
//   chain    GEMVER → BiCGK → GEMVER wired as the Chain system (systems.hpp:214-266), or the crafted chain's three
//            groups (systems.hpp:269-330)                                          → cspb_gemver_chain
//   NS       the 19 stages of NsFused or the 18 components of NsUnfused (examples/ns-residual/systems.hpp:31-140,
//            components.hpp:100-852), either limiter and boundary  → cspb_ns_compressible, whose 18 diagnostics
//            are then copied into the Dt, Ws, Sq, Det and Err variables
//
// The kernel writes the run's outputs (B, x, w; q, s); the partial-sum variables between the run's components (P, Pq,
// Ps) are not written, so a run whose partials something else reads, or whose scale is itself computed, is left to
// the generic path. The scales (the reference's `scale` inputs: α = β = 1/√n in the chain) are read from their device
// variables once per initialisation. NAGA_COSPAN_GENERIC set in the environment turns every fast path off.
//
// Types and wiring say what a run is built from, not what its bodies compute: a user component with the reference's
// type name and ports could do other arithmetic. So the first forward of every recognised run executes the bodies,
// then the kernel, and compares the outputs the kernel writes (verify_pattern, tolerances kTol*); the kernel replaces
// the bodies only when they agree, and otherwise the bodies' results are kept and the bodies run from then on.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "cspb.h"
#include "model.hpp"

namespace naga::cospan::detail {

// "gc::ColReduce<true>" -> "ColReduce<true>"
inline std::string short_type(const ComponentBase* c) {
    const std::string& t = c->type_name_;
    const std::size_t lt = t.find('<');
    const std::size_t cut = t.rfind("::", lt == std::string::npos ? std::string::npos : lt);
    return cut == std::string::npos ? t : t.substr(cut + 2);
}

inline bool has_port(const ComponentBase* c, const char* name) {
    for (auto& p : c->ports_)
        if (p.name == name) return true;
    return false;
}

struct PatternLeaves {
    std::vector<ComponentBase*> comps;  // the components of every leaf, in run order
    std::vector<std::size_t> leaf_of;   // comps[i] runs in leaf leaf_of[i]
    std::vector<std::size_t> first;     // the first component of each leaf (leaves.size() + 1 entries)
};

inline PatternLeaves pattern_leaves(Runtime& rt) {
    PatternLeaves L;
    for (std::size_t i = 0; i < rt.leaves.size(); ++i) {
        L.first.push_back(L.comps.size());
        Node* n = rt.leaves[i];
        if (n->kind == Node::Kind::component) {
            L.comps.push_back(static_cast<ComponentBase*>(n));
            L.leaf_of.push_back(i);
        } else {
            for (ComponentBase* c : static_cast<FusedGroupBase*>(n)->stages_) {
                L.comps.push_back(c);
                L.leaf_of.push_back(i);
            }
        }
    }
    L.first.push_back(L.comps.size());
    return L;
}

// The state a fast path keeps: its workspace and the host copies of its scales.
struct FastState {
    std::vector<int> internal;  // the run's partial-sum variables (not written by the kernel)
    void* ws = nullptr;
    std::size_t ws_bytes = 0;
    std::vector<int> scale_vars;
    std::vector<std::uint64_t> scale_version;
    std::vector<float> scale;
    ~FastState() {
        if (ws) cudaFree(ws);
    }
    // false when the host now views one of the partials (the generic path writes them)
    bool partials_unviewed(const Runtime& rt) const {
        for (auto& v : rt.views)
            for (int iv : internal)
                if (v->var == iv) return false;
        return true;
    }
    void* workspace(Runtime& rt, std::size_t bytes) {
        if (bytes > ws_bytes) {
            if (ws) cudaFree(ws);
            ws = nullptr;
            ++rt.allocs;
            cuda_check(cudaMalloc(&ws, bytes), "fast-path workspace");
            ws_bytes = bytes;
        }
        return ws;
    }
    // the current value of every scale variable (a device read only after an initializer wrote it again)
    void refresh(Runtime& rt) {
        for (std::size_t k = 0; k < scale_vars.size(); ++k) {
            Var& v = rt.vars[std::size_t(scale_vars[k])];
            if (v.version == scale_version[k]) continue;
            float h = 0.f;
            ++rt.host_syncs;
            cuda_check(cudaStreamSynchronize(rt.stream), "scale");
            cuda_check(cudaMemcpy(&h, v.data, sizeof(float), cudaMemcpyDeviceToHost), "scale");
            scale[k] = h;
            scale_version[k] = v.version;
        }
    }
};

inline int var_id(Runtime& rt, ComponentBase* c, const char* port) {
    auto it = rt.key_var.find(c->path() + "." + port);
    return it == rt.key_var.end() ? -1 : it->second;
}

// Whether a component outside `run` touches one of the `internal` variables (host views are checked at run time).
inline bool internal_escapes(Runtime& rt, const std::vector<ComponentBase*>& run, const std::vector<int>& internal) {
    for (ComponentBase* c : rt.components) {
        bool inside = false;
        for (ComponentBase* r : run) inside = inside || r == c;
        if (inside) continue;
        for (auto& p : c->ports_)
            for (int v : internal)
                if (p.var == v) return true;
    }
    return false;
}

// The leaves [lo, hi] must hold exactly the components comps[a .. a + k).
inline bool whole_leaves(const PatternLeaves& L, std::size_t a, std::size_t k, std::size_t& lo, std::size_t& hi) {
    lo = L.leaf_of[a];
    hi = L.leaf_of[a + k - 1];
    return L.first[lo] == a && L.first[hi + 1] == a + k;
}

inline void fast_fail(int st, const std::string& what) {
    if (st == CSPB_OK) return;
    const std::string m = "naga::cospan: " + what + ": " + cspb_status_string(st);
    if (st == CSPB_ERR_ARGUMENT || st == CSPB_ERR_UNSUPPORTED || st == CSPB_ERR_WORKSPACE || st == CSPB_ERR_TOO_LARGE)
        throw std::invalid_argument(m);
    throw std::runtime_error(m);
}

inline bool scale_is_input(Runtime& rt, int v) {
    return v >= 0 && !rt.vars[std::size_t(v)].produced && rt.vars[std::size_t(v)].dtype == DType::f32;
}

// ---- GEMVER --------------------------------------------------------------------------------------------------------
struct GemverMatch {
    ComponentBase *r2u, *gtp, *cred, *gemv;
    int vB, vP, vbeta, valpha;
};

// comps[a .. a + 4) by type and wiring (the leaf boundaries and escaping partials are checked by the caller)
inline bool match_gemver(Runtime& rt, const PatternLeaves& L, std::size_t a, GemverMatch& m) {
    if (a + 4 > L.comps.size()) return false;
    ComponentBase *r2u = L.comps[a], *gtp = L.comps[a + 1], *cred = L.comps[a + 2], *gemv = L.comps[a + 3];
    const std::string t0 = short_type(r2u), t1 = short_type(gtp);
    if (!(t0 == "Rank2Update" || t0 == "Rank2UpdateLocal") || !(t1 == "GemvTPartial" || t1 == "GemvTPartialLocal") ||
        short_type(cred) != "ColReduce<true>" || short_type(gemv) != "Gemv")
        return false;
    const int vB = var_id(rt, r2u, "B"), vP = var_id(rt, gtp, "P");
    if (vB < 0 || var_id(rt, gemv, "B") != vB || var_id(rt, cred, "P") != vP || var_id(rt, cred, "x") != var_id(rt, gemv, "x"))
        return false;
    if (has_port(gtp, "B") && var_id(rt, gtp, "B") != vB) return false;  // the local variant takes B from its tile
    const int vbeta = var_id(rt, cred, "scale"), valpha = var_id(rt, gemv, "scale");
    if (!scale_is_input(rt, vbeta) || !scale_is_input(rt, valpha)) return false;
    m = GemverMatch{r2u, gtp, cred, gemv, vB, vP, vbeta, valpha};
    return true;
}

// cspb_gemver_fused over a matched run, with its scales β and α
inline void launch_gemver(Runtime& rt, FastState& st, const GemverMatch& g, std::int64_t n, float beta, float alpha) {
    cspb_gemver_desc d{};
    d.n = n;
    d.lda = n;
    d.ldb = n;
    d.a_dtype = CSPB_F32;
    d.A = rt.var_of_port(g.r2u, "A").data;
    d.u1 = static_cast<const float*>(rt.var_of_port(g.r2u, "u1").data);
    d.v1 = static_cast<const float*>(rt.var_of_port(g.r2u, "v1").data);
    d.u2 = static_cast<const float*>(rt.var_of_port(g.r2u, "u2").data);
    d.v2 = static_cast<const float*>(rt.var_of_port(g.r2u, "v2").data);
    d.y = static_cast<const float*>(rt.var_of_port(g.gtp, "y").data);
    d.z = static_cast<const float*>(rt.var_of_port(g.cred, "z").data);
    d.beta = beta;
    d.alpha = alpha;
    d.B = static_cast<float*>(rt.var_of_port(g.r2u, "B").data);
    d.x = static_cast<float*>(rt.var_of_port(g.cred, "x").data);
    d.w = static_cast<float*>(rt.var_of_port(g.gemv, "y").data);
    d.workspace_bytes = cspb_gemver_workspace_bytes(n);
    d.workspace = st.workspace(rt, d.workspace_bytes);
    if (rt.trace)
        std::fprintf(stderr, "[cospan] fast path cspb_gemver_fused n=%lld for '%s' .. '%s'\n", (long long)n,
                     g.r2u->path().c_str(), g.gemv->path().c_str());
    fast_fail(cspb_gemver_fused(&d, rt.stream), "'" + g.r2u->path() + "' (GEMVER fast path)");
}

// the square matrix a GEMVER run reads (0: not square)
inline std::int64_t gemver_n(Runtime& rt, const GemverMatch& g) {
    Var& A = rt.var_of_port(g.r2u, "A");
    return (A.rank == 2 && A.shape[0] == A.shape[1]) ? std::int64_t(A.shape[0]) : 0;
}

// Tolerances of a fast path's outputs against the components' own bodies (relative L2). Two f32 evaluations that
// round differently (the bodies compile with fused multiply-adds, the kernels round each operation of Â; sums in
// another order) stay well inside them: Â about 1e-7, x and w about 1e-7 at n = 16384, an NS residual about 2e-5 at
// 4096². A component that computes something else differs at O(1).
constexpr double kTolMatrix = 1e-6, kTolVector = 1e-5, kTolField = 1e-4;

// Σ (a - b)², Σ b² and the number of positions where b is finite and a is not, in f64, one atomic per block.
template <int kUnused = 0>
__global__ void k_fast_check(const float* a, const float* b, std::size_t n, double* acc) {
    double d = 0.0, s = 0.0, bad = 0.0;
    for (std::size_t i = std::size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += std::size_t(gridDim.x) * blockDim.x) {
        const float x = a[i], y = b[i];
        if (isfinite(y) && !isfinite(x)) bad += 1.0;
        const double t = double(x) - double(y);
        d += t * t;
        s += double(y) * double(y);
    }
    for (int off = 16; off >= 1; off >>= 1) {
        d += __shfl_xor_sync(0xffffffffu, d, off);
        s += __shfl_xor_sync(0xffffffffu, s, off);
        bad += __shfl_xor_sync(0xffffffffu, bad, off);
    }
    __shared__ double r[3][32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { r[0][w] = d; r[1][w] = s; r[2][w] = bad; }
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (int k = 0; k < int(blockDim.x >> 5); ++k) t += r[threadIdx.x][k];
        atomicAdd(acc + threadIdx.x, t);
    }
}

// Runs pattern `pat`'s kernel after the components' own bodies wrote its outputs, and compares. 1: every output within
// its tolerance (the kernel runs from now on); -1: an output differs, the bodies' values are put back and the bodies
// run from now on (a component with the same type name and wiring but other arithmetic is never replaced); 0: the fast
// path declined this forward (checked again on the next).
inline int verify_pattern(Runtime& rt, std::size_t pat) {
    const auto& checks = rt.pattern_checks[pat];
    std::vector<void*> snap(checks.size(), nullptr);
    std::vector<std::size_t> count(checks.size(), 0);
    for (std::size_t k = 0; k < checks.size(); ++k) {
        Var& v = rt.vars[std::size_t(checks[k].first)];
        if (v.dtype != DType::f32 || !v.data || v.elements() == 0) continue;
        count[k] = v.elements();
        ++rt.allocs;
        cuda_check(cudaMalloc(&snap[k], count[k] * sizeof(float)), "fast-path check");
        cuda_check(cudaMemcpyAsync(snap[k], v.data, count[k] * sizeof(float), cudaMemcpyDeviceToDevice, rt.stream),
                   "fast-path check");
    }
    std::size_t next = 0;
    int result = 0;
    if (rt.pattern_runs[pat](rt, next)) {
        double* acc = nullptr;
        ++rt.allocs;
        cuda_check(cudaMalloc(&acc, 3 * sizeof(double) * checks.size()), "fast-path check");
        cuda_check(cudaMemsetAsync(acc, 0, 3 * sizeof(double) * checks.size(), rt.stream), "fast-path check");
        for (std::size_t k = 0; k < checks.size(); ++k) {
            if (!snap[k]) continue;
            const float* fast = static_cast<const float*>(rt.vars[std::size_t(checks[k].first)].data);
            const unsigned blocks = unsigned(std::min<std::size_t>((count[k] + 255) / 256, 1024));
            k_fast_check<<<blocks, 256, 0, rt.stream>>>(fast, static_cast<const float*>(snap[k]), count[k], acc + 3 * k);
        }
        std::vector<double> h(3 * checks.size(), 0.0);
        ++rt.host_syncs;
        cuda_check(cudaMemcpyAsync(h.data(), acc, h.size() * sizeof(double), cudaMemcpyDeviceToHost, rt.stream),
                   "fast-path check");
        cuda_check(cudaStreamSynchronize(rt.stream), "fast-path check");
        cudaFree(acc);
        result = 1;
        std::string bad;
        for (std::size_t k = 0; k < checks.size(); ++k) {
            if (!snap[k]) continue;
            const double d = h[3 * k], s2 = h[3 * k + 1], nonfinite = h[3 * k + 2];
            const double rel = s2 > 0.0 ? std::sqrt(d / s2) : (d > 0.0 ? 1.0 : 0.0);
            if (nonfinite > 0.0 || !(rel <= checks[k].second)) {
                result = -1;
                bad += " '" + rt.vars[std::size_t(checks[k].first)].name + "' (relative L2 " + std::to_string(rel) + ")";
            }
        }
        if (result < 0) {
            for (std::size_t k = 0; k < checks.size(); ++k)
                if (snap[k])
                    cuda_check(cudaMemcpyAsync(rt.vars[std::size_t(checks[k].first)].data, snap[k],
                                               count[k] * sizeof(float), cudaMemcpyDeviceToDevice, rt.stream),
                               "fast-path check");
            std::fprintf(stderr, "[cospan] fast path %zu not used: the kernel and the components' own bodies differ in%s;"
                                 " the bodies run\n", pat, bad.c_str());
        } else if (rt.trace) {
            std::fprintf(stderr, "[cospan] fast path %zu agrees with the components' own bodies\n", pat);
        }
    }
    cuda_check(cudaStreamSynchronize(rt.stream), "fast-path check");
    for (void* p : snap)
        if (p) cudaFree(p);
    return result;
}

inline void claim(Runtime& rt, int pat, std::size_t lo, std::size_t hi,
                  std::vector<std::pair<int, double>> checks) {
    rt.pattern_checks.push_back(std::move(checks));
    rt.pattern_verified.push_back(0);
    rt.pattern_hi.push_back(hi);
    rt.pattern_at[lo] = pat;
    for (std::size_t i = lo + 1; i <= hi; ++i) rt.pattern_at[i] = -2;
}

inline bool try_gemver(Runtime& rt, const PatternLeaves& L, std::size_t a) {
    GemverMatch g;
    if (!match_gemver(rt, L, a, g)) return false;
    std::size_t lo, hi;
    if (!whole_leaves(L, a, 4, lo, hi)) return false;
    if (internal_escapes(rt, {g.r2u, g.gtp, g.cred, g.gemv}, {g.vP})) return false;

    auto st = std::make_shared<FastState>();
    st->internal = {g.vP};
    st->scale_vars = {g.vbeta, g.valpha};
    st->scale_version = {~0ull, ~0ull};
    st->scale = {0.f, 0.f};
    rt.pattern_state.push_back(st);
    const int pat = int(rt.pattern_runs.size());
    rt.pattern_runs.push_back([st, g](Runtime& rt, std::size_t&) {
        if (!st->partials_unviewed(rt)) return false;
        for (ComponentBase* c : {g.r2u, g.gtp, g.cred, g.gemv}) rt.prepare(c);
        const std::int64_t n = gemver_n(rt, g);
        if (n == 0) return false;
        st->refresh(rt);
        launch_gemver(rt, *st, g, n, st->scale[0], st->scale[1]);
        return true;
    });
    claim(rt, pat, lo, hi, {{g.vB, kTolMatrix}, {var_id(rt, g.cred, "x"), kTolVector}, {var_id(rt, g.gemv, "y"), kTolVector}});
    return true;
}

// ---- BiCGK ---------------------------------------------------------------------------------------------------------
struct BicgkMatch {
    ComponentBase *c0, *c1, *c2;
    int vB, vp, vr, vq, vs, vscale_s, vscale_q;  // vscale_q: -1 for the one-pass form (no scale on q)
    std::vector<int> internal;
};

inline bool match_bicgk(Runtime& rt, const PatternLeaves& L, std::size_t a, BicgkMatch& m) {
    if (a + 3 > L.comps.size()) return false;
    ComponentBase *c0 = L.comps[a], *c1 = L.comps[a + 1], *c2 = L.comps[a + 2];
    if (short_type(c2) != "ColReduce<false>") return false;
    const std::string t0 = short_type(c0), t1 = short_type(c1);
    int vB, vp, vr, vq, vscale_q = -1;
    std::vector<int> internal;
    if (t0 == "BicgkOnePass" && t1 == "RowReduce") {
        vB = var_id(rt, c0, "B");
        vp = var_id(rt, c0, "p");
        vr = var_id(rt, c0, "r");
        if (var_id(rt, c1, "Pq") != var_id(rt, c0, "Pq") || var_id(rt, c2, "P") != var_id(rt, c0, "Ps")) return false;
        vq = var_id(rt, c1, "q");
        internal = {var_id(rt, c0, "Pq"), var_id(rt, c0, "Ps")};
    } else if (t0 == "Gemv" && t1 == "GemvTPartial") {
        vB = var_id(rt, c0, "B");
        if (var_id(rt, c1, "B") != vB || var_id(rt, c2, "P") != var_id(rt, c1, "P")) return false;
        vp = var_id(rt, c0, "x");
        vr = var_id(rt, c1, "y");
        vq = var_id(rt, c0, "y");
        vscale_q = var_id(rt, c0, "scale");
        internal = {var_id(rt, c1, "P")};
        if (!scale_is_input(rt, vscale_q)) return false;
    } else {
        return false;
    }
    const int vs = var_id(rt, c2, "x");
    const int vscale_s = var_id(rt, c2, "scale");
    if (vB < 0 || vp < 0 || vr < 0 || vq < 0 || vs < 0 || !scale_is_input(rt, vscale_s)) return false;
    m = BicgkMatch{c0, c1, c2, vB, vp, vr, vq, vs, vscale_s, vscale_q, internal};
    return true;
}

// the BiCGK run's scale variables, s's first
inline std::vector<int> bicgk_scales(const BicgkMatch& m) {
    std::vector<int> v{m.vscale_s};
    if (m.vscale_q >= 0) v.push_back(m.vscale_q);
    return v;
}

inline void launch_bicgk(Runtime& rt, FastState& st, const BicgkMatch& m, std::int64_t n) {
    cspb_bicgk_desc d{};
    d.n = n;
    d.ldb = n;
    d.b_dtype = CSPB_F32;
    d.B = rt.vars[std::size_t(m.vB)].data;
    d.p = static_cast<const float*>(rt.vars[std::size_t(m.vp)].data);
    d.r = static_cast<const float*>(rt.vars[std::size_t(m.vr)].data);
    d.q = static_cast<float*>(rt.vars[std::size_t(m.vq)].data);
    d.s = static_cast<float*>(rt.vars[std::size_t(m.vs)].data);
    d.workspace_bytes = cspb_bicgk_workspace_bytes(n);
    d.workspace = st.workspace(rt, d.workspace_bytes);
    if (rt.trace)
        std::fprintf(stderr, "[cospan] fast path cspb_bicgk_fused n=%lld for '%s' .. '%s'\n", (long long)n,
                     m.c0->path().c_str(), m.c2->path().c_str());
    fast_fail(cspb_bicgk_fused(&d, rt.stream), "'" + m.c0->path() + "' (BiCGK fast path)");
}

inline bool try_bicgk(Runtime& rt, const PatternLeaves& L, std::size_t a) {
    BicgkMatch m;
    if (!match_bicgk(rt, L, a, m)) return false;
    std::size_t lo, hi;
    if (!whole_leaves(L, a, 3, lo, hi)) return false;
    if (internal_escapes(rt, {m.c0, m.c1, m.c2}, m.internal)) return false;

    auto st = std::make_shared<FastState>();
    st->internal = m.internal;
    st->scale_vars = bicgk_scales(m);
    st->scale_version.assign(st->scale_vars.size(), ~0ull);
    st->scale.assign(st->scale_vars.size(), 0.f);
    rt.pattern_state.push_back(st);
    const int pat = int(rt.pattern_runs.size());
    rt.pattern_runs.push_back([st, m](Runtime& rt, std::size_t&) {
        if (!st->partials_unviewed(rt)) return false;
        for (ComponentBase* c : {m.c0, m.c1, m.c2}) rt.prepare(c);
        st->refresh(rt);
        for (float s : st->scale)
            if (s != 1.0f) return false;  // the kernel forms q = B·p and s = Bᵀ·r unscaled
        Var& B = rt.vars[std::size_t(m.vB)];
        if (B.rank != 2 || B.shape[0] != B.shape[1]) return false;
        launch_bicgk(rt, *st, m, std::int64_t(B.shape[0]));
        return true;
    });
    claim(rt, pat, lo, hi, {{m.vq, kTolVector}, {m.vs, kTolVector}});
    return true;
}

// ---- the gemver chain ----------------------------------------------------------------------------------------------
// The variables cspb_gemver_chain reads and writes, by id (their device pointers are taken at run time).
struct ChainVars {
    int A0, u1a, v1a, u2a, v2a, ya, za, u1b, v1b, u2b, v2b, B1, x1, w1, q, s, B2, x2, w2;
    bool valid() const {
        for (int v : {A0, u1a, v1a, u2a, v2a, ya, za, u1b, v1b, u2b, v2b, B1, x1, w1, q, s, B2, x2, w2})
            if (v < 0) return false;
        return true;
    }
};

// the outputs a chain kernel writes
inline std::vector<std::pair<int, double>> chain_checks(const ChainVars& c) {
    return {{c.B1, kTolMatrix}, {c.x1, kTolVector}, {c.w1, kTolVector}, {c.q, kTolVector}, {c.s, kTolVector},
            {c.B2, kTolMatrix}, {c.x2, kTolVector}, {c.w2, kTolVector}};
}

inline void launch_chain(Runtime& rt, FastState& st, const ChainVars& c, std::int64_t n, float alpha, float beta,
                         const ComponentBase* first, const ComponentBase* last) {
    auto f = [&](int v) { return static_cast<float*>(rt.vars[std::size_t(v)].data); };
    cspb_chain_desc d{};
    d.n = n;
    d.A0 = f(c.A0);
    d.u1a = f(c.u1a); d.v1a = f(c.v1a); d.u2a = f(c.u2a); d.v2a = f(c.v2a);
    d.ya = f(c.ya);
    d.za = f(c.za);
    d.u1b = f(c.u1b); d.v1b = f(c.v1b); d.u2b = f(c.u2b); d.v2b = f(c.v2b);
    d.alpha = alpha;
    d.beta = beta;
    d.B1 = f(c.B1); d.x1 = f(c.x1); d.w1 = f(c.w1);
    d.q = f(c.q); d.s = f(c.s);
    d.B2 = f(c.B2); d.x2 = f(c.x2); d.w2 = f(c.w2);
    d.workspace_bytes = cspb_chain_workspace_bytes(n);
    d.workspace = st.workspace(rt, d.workspace_bytes);
    if (rt.trace)
        std::fprintf(stderr, "[cospan] fast path cspb_gemver_chain n=%lld for '%s' .. '%s'\n", (long long)n,
                     first->path().c_str(), last->path().c_str());
    fast_fail(cspb_gemver_chain(&d, rt.stream), "'" + first->path() + "' (gemver chain fast path)");
}

// G1's side of the chain's variables (a matched GEMVER run)
inline void chain_g1_vars(Runtime& rt, const GemverMatch& g1, ChainVars& c) {
    c.A0 = var_id(rt, g1.r2u, "A");
    c.u1a = var_id(rt, g1.r2u, "u1"); c.v1a = var_id(rt, g1.r2u, "v1");
    c.u2a = var_id(rt, g1.r2u, "u2"); c.v2a = var_id(rt, g1.r2u, "v2");
    c.ya = var_id(rt, g1.gtp, "y");
    c.za = var_id(rt, g1.cred, "z");
    c.B1 = g1.vB;
    c.x1 = var_id(rt, g1.cred, "x");
    c.w1 = var_id(rt, g1.gemv, "y");
}

// A GEMVER run, a BiCGK run and a GEMVER run, wired as the reference's Chain system (systems.hpp:214-266): BiCGK's B,
// p, r are G1's B, x, w, and G2's A, y, z are G1's B and BiCGK's q, s. cspb_gemver_chain does the three in six matrix
// passes (two launches) instead of the single kernels' eight. It takes one α and one β for both GEMVERs, as the
// reference's chain ties them; if G1's and G2's scales differ at run time, the fast path runs the three single
// kernels instead.
inline bool try_chain(Runtime& rt, const PatternLeaves& L, std::size_t a) {
    GemverMatch g1, g2;
    BicgkMatch bk;
    if (!match_gemver(rt, L, a, g1) || !match_bicgk(rt, L, a + 4, bk) || !match_gemver(rt, L, a + 7, g2)) return false;
    if (bk.vB != g1.vB || bk.vp != var_id(rt, g1.cred, "x") || bk.vr != var_id(rt, g1.gemv, "y")) return false;
    if (var_id(rt, g2.r2u, "A") != g1.vB || var_id(rt, g2.gtp, "y") != bk.vq || var_id(rt, g2.cred, "z") != bk.vs)
        return false;
    ChainVars cv;
    chain_g1_vars(rt, g1, cv);
    cv.u1b = var_id(rt, g2.r2u, "u1"); cv.v1b = var_id(rt, g2.r2u, "v1");
    cv.u2b = var_id(rt, g2.r2u, "u2"); cv.v2b = var_id(rt, g2.r2u, "v2");
    cv.q = bk.vq;
    cv.s = bk.vs;
    cv.B2 = g2.vB;
    cv.x2 = var_id(rt, g2.cred, "x");
    cv.w2 = var_id(rt, g2.gemv, "y");
    if (!cv.valid()) return false;
    std::size_t lo, hi;
    if (!whole_leaves(L, a, 11, lo, hi)) return false;
    std::vector<int> internal = bk.internal;
    internal.push_back(g1.vP);
    internal.push_back(g2.vP);
    if (internal_escapes(rt, {g1.r2u, g1.gtp, g1.cred, g1.gemv, bk.c0, bk.c1, bk.c2, g2.r2u, g2.gtp, g2.cred, g2.gemv},
                         internal))
        return false;

    auto st = std::make_shared<FastState>();
    st->internal = internal;
    st->scale_vars = {g1.vbeta, g1.valpha, g2.vbeta, g2.valpha};  // then BiCGK's
    for (int v : bicgk_scales(bk)) st->scale_vars.push_back(v);
    st->scale_version.assign(st->scale_vars.size(), ~0ull);
    st->scale.assign(st->scale_vars.size(), 0.f);
    rt.pattern_state.push_back(st);
    const int pat = int(rt.pattern_runs.size());
    rt.pattern_runs.push_back([st, g1, bk, g2, cv](Runtime& rt, std::size_t&) {
        if (!st->partials_unviewed(rt)) return false;
        for (ComponentBase* c : {g1.r2u, g1.gtp, g1.cred, g1.gemv, bk.c0, bk.c1, bk.c2, g2.r2u, g2.gtp, g2.cred, g2.gemv})
            rt.prepare(c);
        const std::int64_t n = gemver_n(rt, g1);
        if (n == 0) return false;
        st->refresh(rt);
        for (std::size_t k = 4; k < st->scale.size(); ++k)
            if (st->scale[k] != 1.0f) return false;  // BiCGK forms q = B·p and s = Bᵀ·r unscaled
        const float beta1 = st->scale[0], alpha1 = st->scale[1], beta2 = st->scale[2], alpha2 = st->scale[3];
        if (beta1 != beta2 || alpha1 != alpha2) {
            // one workspace size for the three (no reallocation between them)
            st->workspace(rt, std::max(cspb_gemver_workspace_bytes(n), cspb_bicgk_workspace_bytes(n)));
            launch_gemver(rt, *st, g1, n, beta1, alpha1);
            launch_bicgk(rt, *st, bk, n);
            launch_gemver(rt, *st, g2, n, beta2, alpha2);
            return true;
        }
        launch_chain(rt, *st, cv, n, alpha1, beta1, g1.r2u, g2.gemv);
        return true;
    });
    claim(rt, pat, lo, hi, chain_checks(cv));
    return true;
}

// The crafted chain (systems.hpp:269-330): G1 as a GEMVER run; a middle group in which BicgkTileLocal reads each B1
// tile once for q's and s's partials and Rank2UpdateFromLocal forms B2 from the same tile, then RowReduce → q and
// ColReduce<false> → s; and G2 without its update (GemvTPartial → ColReduce<true> → Gemv over B2). The same six-pass
// kernel computes it. The middle group's scale on s must be 1 and both GEMVERs' scales equal; otherwise the run keeps
// its own bodies.
inline bool try_crafted_chain(Runtime& rt, const PatternLeaves& L, std::size_t a) {
    GemverMatch g1;
    if (a + 11 > L.comps.size() || !match_gemver(rt, L, a, g1)) return false;
    ComponentBase *bk = L.comps[a + 4], *r2u = L.comps[a + 5], *rowred = L.comps[a + 6], *creds = L.comps[a + 7];
    ComponentBase *gtp = L.comps[a + 8], *cred = L.comps[a + 9], *gemv = L.comps[a + 10];
    if (short_type(bk) != "BicgkTileLocal" || short_type(r2u) != "Rank2UpdateFromLocal" ||
        short_type(rowred) != "RowReduce" || short_type(creds) != "ColReduce<false>" ||
        short_type(gtp) != "GemvTPartial" || short_type(cred) != "ColReduce<true>" || short_type(gemv) != "Gemv")
        return false;
    if (L.leaf_of[a + 5] != L.leaf_of[a + 4]) return false;  // the update reads the tile BicgkTileLocal loaded
    const int vPq = var_id(rt, bk, "Pq"), vPs = var_id(rt, bk, "Ps"), vP2 = var_id(rt, gtp, "P");
    ChainVars cv;
    chain_g1_vars(rt, g1, cv);
    if (var_id(rt, bk, "B") != g1.vB || var_id(rt, bk, "p") != cv.x1 || var_id(rt, bk, "r") != cv.w1) return false;
    if (var_id(rt, rowred, "Pq") != vPq || var_id(rt, creds, "P") != vPs) return false;
    cv.u1b = var_id(rt, r2u, "u1"); cv.v1b = var_id(rt, r2u, "v1");
    cv.u2b = var_id(rt, r2u, "u2"); cv.v2b = var_id(rt, r2u, "v2");
    cv.q = var_id(rt, rowred, "q");
    cv.s = var_id(rt, creds, "x");
    cv.B2 = var_id(rt, r2u, "B");
    cv.x2 = var_id(rt, cred, "x");
    cv.w2 = var_id(rt, gemv, "y");
    if (!cv.valid()) return false;
    if (var_id(rt, gtp, "B") != cv.B2 || var_id(rt, gtp, "y") != cv.q || var_id(rt, cred, "P") != vP2 ||
        var_id(rt, cred, "z") != cv.s || var_id(rt, gemv, "B") != cv.B2 || var_id(rt, gemv, "x") != cv.x2)
        return false;
    const int vscale_s = var_id(rt, creds, "scale"), vbeta2 = var_id(rt, cred, "scale"), valpha2 = var_id(rt, gemv, "scale");
    if (!scale_is_input(rt, vscale_s) || !scale_is_input(rt, vbeta2) || !scale_is_input(rt, valpha2)) return false;
    std::size_t lo, hi;
    if (!whole_leaves(L, a, 11, lo, hi)) return false;
    const std::vector<ComponentBase*> run{g1.r2u, g1.gtp, g1.cred, g1.gemv, bk, r2u, rowred, creds, gtp, cred, gemv};
    const std::vector<int> internal{g1.vP, vPq, vPs, vP2};
    if (internal_escapes(rt, run, internal)) return false;

    auto st = std::make_shared<FastState>();
    st->internal = internal;
    st->scale_vars = {g1.vbeta, g1.valpha, vbeta2, valpha2, vscale_s};
    st->scale_version.assign(st->scale_vars.size(), ~0ull);
    st->scale.assign(st->scale_vars.size(), 0.f);
    rt.pattern_state.push_back(st);
    const int pat = int(rt.pattern_runs.size());
    rt.pattern_runs.push_back([st, g1, run, cv](Runtime& rt, std::size_t&) {
        if (!st->partials_unviewed(rt)) return false;
        for (ComponentBase* c : run) rt.prepare(c);
        const std::int64_t n = gemver_n(rt, g1);
        if (n == 0) return false;
        st->refresh(rt);
        const float beta1 = st->scale[0], alpha1 = st->scale[1], beta2 = st->scale[2], alpha2 = st->scale[3];
        if (st->scale[4] != 1.0f || beta1 != beta2 || alpha1 != alpha2) return false;
        launch_chain(rt, *st, cv, n, alpha1, beta1, run.front(), run.back());
        return true;
    });
    claim(rt, pat, lo, hi, chain_checks(cv));
    return true;
}

// ---- NS residual (compressible) ------------------------------------------------------------------------------------
// A stage's role: its type with the limiter / boundary argument dropped ("Reconstruct<nsr::MinMod>" -> "Reconstruct<>").
inline std::string ns_role(const ComponentBase* c, int& lim, int& walls) {
    std::string t = short_type(c);
    const std::size_t lt = t.find('<');
    if (lt != std::string::npos) {
        const std::string arg = t.substr(lt + 1);
        if (arg.find("MinMod") != std::string::npos) { lim = 0; return t.substr(0, lt) + "<>"; }
        if (arg.find("VanLeer") != std::string::npos) { lim = 1; return t.substr(0, lt) + "<>"; }
        if (arg.find("BcWalls") != std::string::npos) { walls = 1; return t.substr(0, lt) + "<>"; }
        if (arg.find("BcPeriodic") != std::string::npos) { walls = 0; return t.substr(0, lt) + "<>"; }
    }
    return t;
}

inline bool try_ns(Runtime& rt, const PatternLeaves& L, std::size_t a) {
    static const std::vector<std::string> fused = {
        "InitDiagnostics", "LoadTile", "ApplyBoundary<>", "ToPrimitive", "Gradients", "Reconstruct<>", "ConvFlux<0>",
        "ConvFlux<1>", "ViscFlux<0>", "ViscFlux<1>", "ConvDivergence<true>", "ViscDivergence", "LocalTimestep<true>",
        "WaveSpeed<true>", "ResidualSquares<true>", "DetNorm", "DetExtreme<true>", "DetExtreme<false>",
        "ErrorStage<true>"};
    static const std::vector<std::string> unfused = {
        "InitDiagnostics", "PadBoundary<>", "ToPrimitiveG", "GradientsG", "ReconstructG<>", "ConvFluxG<0>",
        "ConvFluxG<1>", "ViscFluxG<0>", "ViscFluxG<1>", "ConvDivergence<false>", "ViscDivergenceChained",
        "LocalTimestep<false>", "WaveSpeed<false>", "ResidualSquares<false>", "DetNorm", "DetExtreme<true>",
        "DetExtreme<false>", "ErrorStage<false>"};
    int lim = -1, walls = -1;
    for (const auto* fam : {&fused, &unfused}) {
        const std::size_t k = fam->size();
        if (a + k > L.comps.size()) continue;
        std::vector<std::string> got;
        std::vector<ComponentBase*> run(L.comps.begin() + std::ptrdiff_t(a), L.comps.begin() + std::ptrdiff_t(a + k));
        for (ComponentBase* c : run) got.push_back(ns_role(c, lim, walls));
        std::vector<std::string> want = *fam;
        std::sort(got.begin(), got.end());
        std::sort(want.begin(), want.end());
        if (got != want || lim < 0 || walls < 0) continue;
        std::size_t lo, hi;
        if (!whole_leaves(L, a, k, lo, hi)) return false;
        auto find = [&](const std::string& role) -> ComponentBase* {
            int l2 = lim, w2 = walls;
            for (ComponentBase* c : run)
                if (ns_role(c, l2, w2) == role) return c;
            return nullptr;
        };
        ComponentBase* init = find("InitDiagnostics");
        ComponentBase* load = find(fam == &fused ? "LoadTile" : "PadBoundary<>");
        ComponentBase* vdiv = find(fam == &fused ? "ViscDivergence" : "ViscDivergenceChained");
        ComponentBase* detn = find("DetNorm");
        ComponentBase* detd = find("DetExtreme<true>");
        ComponentBase* detw = find("DetExtreme<false>");
        ComponentBase* err = find(fam == &fused ? "ErrorStage<true>" : "ErrorStage<false>");
        const int vU = var_id(rt, load, "U"), vR = var_id(rt, vdiv, "R");
        const std::vector<int> outs = {var_id(rt, init, "Dt"), var_id(rt, init, "Ws"), var_id(rt, init, "Sq"),
                                       var_id(rt, detn, "Det"), var_id(rt, detd, "Det"), var_id(rt, detw, "Det"),
                                       var_id(rt, err, "Err")};
        if (vU < 0 || vR < 0) return false;
        for (int v : outs)
            if (v < 0) return false;
        // every other variable the run touches is internal (fluxes, primitives, partials): nothing else may use it
        std::vector<int> internal;
        for (ComponentBase* c : run)
            for (auto& pr : c->ports_) {
                const int v = pr.var;
                bool keep = v == vU || v == vR || var_id(rt, c, "geo") == v;
                for (int o : outs) keep = keep || o == v;
                if (!keep && std::find(internal.begin(), internal.end(), v) == internal.end()) internal.push_back(v);
            }
        if (internal_escapes(rt, run, internal)) return false;

        auto st = std::make_shared<FastState>();
        st->internal = internal;
        rt.pattern_state.push_back(st);
        const int pat = int(rt.pattern_runs.size());
        rt.pattern_runs.push_back([st, run, vU, vR, outs, lim, walls](Runtime& rt, std::size_t&) {
            if (!st->partials_unviewed(rt)) return false;
            for (ComponentBase* c : run) rt.prepare(c);
            Var& U = rt.vars[std::size_t(vU)];
            Var& R = rt.vars[std::size_t(vR)];
            if (U.rank != 3 || U.shape[0] != 4 || R.rank != 3 || R.shape != U.shape) return false;
            const int ny = int(U.shape[1]), nx = int(U.shape[2]);
            const std::size_t wsb = cspb_ns_comp_workspace_bytes(nx, ny);
            // the kernel's workspace, then its 18 diagnostics
            char* ws = static_cast<char*>(st->workspace(rt, (wsb + 255) / 256 * 256 + 256));
            float* diag = reinterpret_cast<float*>(ws + (wsb + 255) / 256 * 256);
            cspb_ns_comp_desc d{};
            d.nx = nx;
            d.ny = ny;
            d.limiter = lim;
            d.walls = walls;
            d.U = static_cast<const float*>(U.data);
            d.R = static_cast<float*>(R.data);
            d.diag = diag;
            d.det_sq64 = nullptr;
            d.workspace = ws;
            d.workspace_bytes = wsb;
            if (rt.trace)
                std::fprintf(stderr, "[cospan] fast path cspb_ns_compressible %dx%d for '%s' .. '%s'\n", nx, ny,
                             run.front()->path().c_str(), run.back()->path().c_str());
            fast_fail(cspb_ns_compressible(&d, rt.stream), "'" + run.front()->path() + "' (NS fast path)");
            // diag: [0] Dt [1] Ws [2..5] Sq | [6..9] detn [10] detd [11] detw | [12..17] Err
            const int at[7] = {0, 1, 2, 6, 10, 11, 12}, len[7] = {1, 1, 4, 4, 1, 1, 6};
            for (int k = 0; k < 7; ++k) {
                Var& o = rt.vars[std::size_t(outs[std::size_t(k)])];
                if (o.elements() != std::size_t(len[k])) throw std::logic_error("naga::cospan: NS fast path: '" + o.name + "' has an unexpected size");
                cuda_check(cudaMemcpyAsync(o.data, diag + at[k], std::size_t(len[k]) * sizeof(float),
                                           cudaMemcpyDeviceToDevice, rt.stream), "NS diagnostics");
            }
            return true;
        });
        // R and the deterministic diagnostics (the atomic ones depend on the order the tiles finish in)
        claim(rt, pat, lo, hi, {{vR, kTolField}, {outs[3], kTolField}, {outs[4], kTolVector}, {outs[5], kTolVector}});
        return true;
    }
    return false;
}

inline void register_patterns(Runtime& rt) {
    rt.pattern_at.assign(rt.leaves.size(), -1);
    rt.pattern_hi.clear();
    rt.pattern_checks.clear();
    rt.pattern_verified.clear();
    if (std::getenv("NAGA_COSPAN_GENERIC")) return;
    const PatternLeaves L = pattern_leaves(rt);
    for (std::size_t a = 0; a < L.comps.size();) {
        if (L.first[L.leaf_of[a]] != a || rt.pattern_at[L.leaf_of[a]] != -1) {  // runs start on a leaf boundary
            ++a;
            continue;
        }
        if (try_chain(rt, L, a) || try_crafted_chain(rt, L, a)) a += 11;
        else if (try_gemver(rt, L, a)) a += 4;
        else if (try_bicgk(rt, L, a)) a += 3;
        else if (try_ns(rt, L, a)) a = L.first[std::size_t(rt.pattern_hi.back()) + 1];
        else ++a;
    }
}

}  // namespace naga::cospan::detail
