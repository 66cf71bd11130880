// naga/cospan/model.hpp — cs::Model and the runtime under it.
//
// Lifecycle (model.hpp:447-532 of the reference): create_model<Root>(args) builds the root System; setup() runs the
// user's setup (children are declared / set up as they are added); the first run() or update_input() finalizes the
// wiring into VARIABLES (one device buffer each: a connect, a tie or a promotion names the same variable); run()
// walks the leaves in declaration order on one CUDA stream — each component's inputs are shaped and materialized
// (allocated, initialized when stale), prepare_forward() shapes its outputs, define_forward() says how it launches —
// and pushes open host views; wait() synchronizes and raises device-side failures.
//
// Leaves whose stages form a chain the cspb library implements as one hand-written kernel (the GEMVER and BiCGK
// stages of the gemver example, the NS fused group of the ns-residual example) run that kernel through the C ABI
// (patterns.hpp); every other leaf runs its own component bodies (component.hpp, system.hpp).
#pragma once

#include <cstdio>
#include <cstdlib>
#include <map>
#include <numeric>
#include <set>

#include "cspb.h"
#include "naga/slabkit/slabkit.hpp"
#include "system.hpp"

namespace naga::cospan {

namespace detail {

inline void cuda_check(cudaError_t e, const std::string& what) {
    if (e != cudaSuccess) throw std::runtime_error("naga::cospan: " + what + ": " + cudaGetErrorString(e));
}

struct ViewState {
    int var = -1;
    void* host = nullptr;
    std::size_t bytes = 0;
    std::array<std::size_t, 4> shape{};
    cudaEvent_t ev = nullptr;
    // a ragged view: N, and the block offsets (a copy of the device column's, or the rows of a dense variable)
    bool ragged = false, per = false;
    std::size_t n = 0, row = 0;
    std::uint32_t* host_offs = nullptr;
    std::uint64_t* host_offs64 = nullptr;  // a column with u64 offsets
    std::size_t offs_cap = 0;
    // block i's start (a column's offsets, u32 or u64, or i rows in)
    std::uint64_t off(std::size_t i) const {
        if (!per) return std::uint64_t(i) * row;
        return host_offs64 ? host_offs64[i] : std::uint64_t(host_offs[i]);
    }
    ~ViewState() {
        if (host) cudaFreeHost(host);
        if (host_offs) cudaFreeHost(host_offs);
        if (host_offs64) cudaFreeHost(host_offs64);
        if (ev) cudaEventDestroy(ev);
    }
};

/// A ragged variable's device counts and block offsets (shape_hook.hpp:215-348 and variable.hpp:252-300 of the
/// reference): N u32 extents and N + 1 offsets, u32 as in the reference (a total below 2^32) or u64 when the hook asks
/// for them (counts_from<std::uint64_t>, built by cspb_build_column64). A counts_from / offsets_from
/// hook builds one with cspb_build_column (one launch; [total, flag] comes back through mapped pinned memory); host
/// counts (a declaration, or a producer's set_shape) are uploaded into one. Shared between variables by set_shape(out,
/// shape_of(in)): the wrappers read the pointers at every bind, so a column that grows is seen by all of them.
struct Column {
    std::uint32_t* ext = nullptr;
    std::uint32_t* offs = nullptr;    // u32 offsets (the default)
    std::uint64_t* offs64 = nullptr;  // u64 offsets, for a column built with wide offsets (counts_from<uint64_t>)
    bool wide = false;
    std::size_t cap = 0;  // entries of offs (ext has at least cap - 1)
    std::size_t n = 0;
    std::uint64_t total = 0;
    std::uint64_t version = 0;
    std::uint32_t* tf = nullptr;  // mapped pinned [total, flag] (u32 offsets) or, as two u64, [total, flag] (u64)
    std::uint32_t* tf_dev = nullptr;
    std::vector<std::size_t> uploaded;  // the host counts in the column (a host column)
    bool has_upload = false;
    std::vector<std::uint32_t> staging;
    std::vector<std::uint64_t> staging64;
    Column() = default;
    Column(const Column&) = delete;
    Column& operator=(const Column&) = delete;
    ~Column() {
        if (ext) cudaFree(ext);
        if (offs) cudaFree(offs);
        if (offs64) cudaFree(offs64);
        if (tf) cudaFreeHost(tf);
    }
    /// Room for n blocks, with u32 or (wide) u64 offsets. A reallocation waits for the stream first (kernels in flight
    /// may read the old arrays).
    void reserve(std::size_t nb, cudaStream_t s, bool want_wide = false) {
        if (!tf) {
            if (cudaHostAlloc(reinterpret_cast<void**>(&tf), 16, cudaHostAllocMapped) != cudaSuccess ||
                cudaHostGetDevicePointer(reinterpret_cast<void**>(&tf_dev), tf, 0) != cudaSuccess)
                throw std::runtime_error("naga::cospan: a ragged column's host word");
        }
        if (nb + 1 <= cap && want_wide == wide) return;
        const std::size_t want = std::max(nb + 1, want_wide == wide ? cap * 2 : nb + 1);
        if (ext || offs || offs64) cudaStreamSynchronize(s);
        if (ext) cudaFree(ext);
        if (offs) cudaFree(offs);
        if (offs64) cudaFree(offs64);
        ext = offs = nullptr;
        offs64 = nullptr;
        wide = want_wide;
        const bool ok = cudaMalloc(&ext, std::max<std::size_t>(want - 1, 1) * 4) == cudaSuccess &&
                        (wide ? cudaMalloc(&offs64, want * 8) : cudaMalloc(&offs, want * 4)) == cudaSuccess;
        if (!ok) throw std::runtime_error("naga::cospan: allocating a ragged column of " + std::to_string(nb) + " blocks");
        cap = want;
    }
};

struct Var {
    int id = -1;
    std::string name;
    DType dtype = DType::f32;
    int rank = -1;
    ShapeSpec spec;                   // what declarations and ties fix
    std::vector<HookDim> hook;        // a shape hook on it
    System* hook_sys = nullptr;
    std::string hook_path;            // the hook's target as its System named it (for messages)
    std::array<std::size_t, 4> shape{};
    bool shape_known = false;
    bool shape_from_prepare = false;  // set by a producer's prepare_forward (re-derived every run)
    void* data = nullptr;
    std::size_t capacity = 0;
    std::optional<InitSpec> init;
    bool stale = false;
    bool produced = false;
    std::uint64_t version = 0;        // incremented whenever an initializer writes the variable
    // ragged (rank 2): N = shape[0], the per-index counts in `column`, `total` elements
    bool ragged_port = false;         // some port on it is a RaggedInput / RaggedOutput
    bool ragged_out = false;          // its producer's port is a RaggedOutput
    bool per = false;                 // its current shape is ragged
    std::uint64_t total = 0;
    std::optional<std::vector<std::size_t>> declared_counts;  // cs::counts / cs::offsets in a declaration
    std::vector<std::size_t> host_counts;                     // counts given on the host (empty for a hooked column)
    std::shared_ptr<Column> column;                           // what its ragged wrappers read
    std::shared_ptr<Column> own_column;                       // where its host counts are uploaded
    std::shared_ptr<Column> hook_column;                      // what its ragged hook builds
    std::size_t elements() const {
        if (per) return std::size_t(total);
        std::size_t n = 1;
        for (int d = 0; d < rank; ++d) n *= shape[d];
        return n;
    }
    std::size_t bytes() const { return elements() * dtype_size(dtype); }
};

struct InitTarget {
    Runtime& rt;
    Var& var;
};

class Runtime {
public:
    cudaStream_t stream = nullptr;
    int device = 0;
    std::uint32_t* ctrl = nullptr;  // 256 bytes: status word, barrier counters
    std::vector<Var> vars;
    std::vector<Node*> leaves;
    std::vector<ComponentBase*> components;  // every component, stages included
    std::vector<std::shared_ptr<ViewState>> views;
    std::unique_ptr<sk::unordered_queue> uq;
    std::map<std::string, int> key_var;      // port / tie key -> variable
    std::map<std::string, std::string> tie_keys;  // system path + "/" + alias -> tie key
    std::vector<std::function<bool(Runtime&, std::size_t&)>> pattern_runs;  // per leaf index: a fast path
    std::vector<int> pattern_at;             // leaf index -> pattern index or -1 (-2: covered, skip)
    std::vector<std::size_t> pattern_hi;     // per pattern: the last leaf it covers
    std::vector<std::shared_ptr<void>> pattern_state;  // what the fast paths keep between runs (workspaces, scales)
    // per pattern: the outputs its kernel writes, each with the relative L2 distance it may keep from the components'
    // own bodies, and whether it was checked against them (0 not yet, 1 agreed: the kernel runs, -1 disagreed: the
    // bodies run)
    std::vector<std::vector<std::pair<int, double>>> pattern_checks;
    std::vector<int> pattern_verified;
    int sms = 0;
    bool trace = false;  // NAGA_COSPAN_TRACE set: every launch and initializer is printed to stderr
    void* scan_ws = nullptr;  // cspb_build_column's workspace (ragged hooks), grown as needed
    std::size_t scan_ws_bytes = 0;
    void* value_buf = nullptr;  // pinned: one element read down by a from_value hook
    // CUDA-graph replay of steady runs (Model::run): a run that made no host wait and no allocation is a template
    // for the next one, which is captured; later runs replay it until an update_input or a new view.
    std::uint64_t host_syncs = 0;  // waits and device reads the host made (hooks, initializers, scale reads, uploads)
    std::uint64_t allocs = 0;      // device allocations
    std::uint64_t epoch = 0;       // bumped by update_input and by a new view
    std::uint64_t steady_epoch = ~0ull;
    std::uint64_t graph_epoch = ~0ull;
    cudaGraphExec_t graph_exec = nullptr;
    bool graph_allowed = true;     // NAGA_COSPAN_NO_GRAPH, NAGA_COSPAN_TRACE or a failed capture turn it off
    std::uint64_t graph_captures = 0, graph_replays = 0;

    Runtime() {
        trace = std::getenv("NAGA_COSPAN_TRACE") != nullptr;
        graph_allowed = !trace && std::getenv("NAGA_COSPAN_NO_GRAPH") == nullptr;
        cuda_check(cudaGetDevice(&device), "cudaGetDevice");
        cuda_check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
        cuda_check(cudaMalloc(&ctrl, 256), "control block");
        cuda_check(cudaMemset(ctrl, 0, 256), "control block");
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        uq = std::make_unique<sk::unordered_queue>(stream);
    }
    ~Runtime() {
        cudaStreamSynchronize(stream);
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        pattern_runs.clear();
        pattern_state.clear();
        pattern_checks.clear();
        for (auto& v : vars)
            if (v.data) cudaFree(v.data);
        if (ctrl) cudaFree(ctrl);
        if (scan_ws) cudaFree(scan_ws);
        if (value_buf) cudaFreeHost(value_buf);
        views.clear();
        uq.reset();
        if (stream) cudaStreamDestroy(stream);
    }

    // ---- shapes and memory ----
    /// A shape hook (shape_hook.hpp:404-527 of the reference): one descriptor per dimension, or one ragged descriptor.
    /// It runs once per forward, when the variable's shape is first needed (Model::run forgets hooked shapes).
    void shape_from_hook(Var& v) {
        if (v.hook.empty()) return;
        const std::string who = "the shape hook on '" + (v.hook_path.empty() ? v.name : v.hook_path) + "'";
        if (v.hook.size() == 1 && (std::holds_alternative<ragged::CountsFrom>(v.hook[0]) ||
                                   std::holds_alternative<ragged::OffsetsFrom>(v.hook[0]))) {
            ragged_hook(v, who);
            return;
        }
        if (int(v.hook.size()) != v.rank)
            throw std::invalid_argument("naga::cospan: " + who + " has " + std::to_string(v.hook.size()) +
                                        " dimensions, the variable has rank " + std::to_string(v.rank));
        if (v.per) v.shape_known = false;  // a dense hook on a variable that was ragged: it is dense now
        v.per = false;
        for (int d = 0; d < v.rank; ++d) {
            const HookDim& h = v.hook[d];
            if (auto f = std::get_if<dim::FixedAtRun>(&h)) v.shape[d] = f->v;
            else if (auto sh = std::get_if<dim::FromShape>(&h)) {
                Var& o = var_of_path(v.hook_sys, sh->path);
                ensure_shape(o);
                if (int(sh->d) >= o.rank)
                    throw std::out_of_range("naga::cospan: " + who + ": '" + sh->path + "' has rank " + std::to_string(o.rank) +
                                            ", no dimension " + std::to_string(sh->d));
                if (o.per && sh->d == 1)
                    throw std::invalid_argument("naga::cospan: " + who + ": dimension 1 of '" + sh->path +
                                                "' is per-index and cannot become a dense dimension (use cs::ragged::counts_from)");
                v.shape[d] = o.shape[sh->d];
            } else if (auto fv = std::get_if<dim::FromValue>(&h)) {
                v.shape[d] = value_of(var_of_path(v.hook_sys, fv->path), fv->path, fv->index, who);
            } else if (auto cu = std::get_if<dim::Custom>(&h)) {
                v.shape[d] = custom_dim(v, *cu);
            } else if (std::holds_alternative<dim::AsIs>(h)) {
                if (!v.shape_known && !(v.spec.rank > d && v.spec.known[d]))
                    throw std::invalid_argument("naga::cospan: '" + v.name + "': as_is on a dimension with no shape");
                if (!v.shape_known) v.shape[d] = v.spec.ext[d];
            } else {
                throw std::invalid_argument("naga::cospan: " + who + ": a ragged descriptor is for a ragged target, as its "
                                            "only descriptor");
            }
        }
        v.shape_known = true;
    }
    std::size_t custom_dim(Var& v, const dim::Custom& c);  // after ShapeHookCtx
    /// The value of element `index` of the integer variable `o`, read down from the device (one small copy, one wait).
    std::size_t value_of(Var& o, const std::string& path, std::size_t index, const std::string& who) {
        const DType dt = value_dtype(o.dtype);
        if (dt == DType::f32 || dt == DType::f64)
            throw std::invalid_argument("naga::cospan: " + who + ": '" + path + "' drives a size by value and must have an "
                                        "integer dtype");
        if (!o.produced) materialize(o);
        ensure_shape(o);
        if (index >= o.elements())
            throw std::invalid_argument("naga::cospan: " + who + ": '" + path + "' drives a size from element " +
                                        std::to_string(index) + " but has only " + std::to_string(o.elements()) + " elements");
        if (!o.data) throw std::logic_error("naga::cospan: " + who + ": '" + path + "' has no data");
        ++host_syncs;
        if (!value_buf) cuda_check(cudaMallocHost(&value_buf, 8), "a hook's value buffer");
        const std::size_t es = dtype_size(dt);
        cuda_check(cudaMemcpyAsync(value_buf, static_cast<const unsigned char*>(o.data) + index * es, es,
                                   cudaMemcpyDeviceToHost, stream), "a hook's value read");
        cuda_check(cudaStreamSynchronize(stream), "a hook's value read");
        std::int64_t val = 0;
        switch (dt) {
            case DType::i32: val = *static_cast<const std::int32_t*>(value_buf); break;
            case DType::u32: val = std::int64_t(*static_cast<const std::uint32_t*>(value_buf)); break;
            case DType::i64: val = *static_cast<const std::int64_t*>(value_buf); break;
            case DType::u64: val = std::int64_t(*static_cast<const std::uint64_t*>(value_buf)); break;
            default: val = *static_cast<const std::uint8_t*>(value_buf); break;
        }
        if (val < 0)
            throw std::invalid_argument("naga::cospan: " + who + ": element " + std::to_string(index) + " of '" + path +
                                        "' is " + std::to_string(val) + "; a size cannot be negative");
        return std::size_t(val);
    }
    /// counts_from / offsets_from: the column is built on the device by cspb_build_column from the source's values
    /// (shape_hook.hpp:215-348 of the reference); only [total, flag] comes back to the host.
    void ragged_hook(Var& v, const std::string& who) {
        if (v.rank != 2) throw std::invalid_argument("naga::cospan: " + who + ": a ragged hook needs a rank-2 target");
        ++host_syncs;
        const bool offsets_mode = std::holds_alternative<ragged::OffsetsFrom>(v.hook[0]);
        const std::string path = offsets_mode ? std::get<ragged::OffsetsFrom>(v.hook[0]).path
                                              : std::get<ragged::CountsFrom>(v.hook[0]).path;
        const bool wide = offsets_mode ? std::get<ragged::OffsetsFrom>(v.hook[0]).wide
                                       : std::get<ragged::CountsFrom>(v.hook[0]).wide;
        Var& src = var_of_path(v.hook_sys, path);
        int code = -1;
        switch (value_dtype(src.dtype)) {
            case DType::i32: code = CSPB_I32; break;
            case DType::u32: code = CSPB_U32; break;
            case DType::i64: code = CSPB_I64; break;
            case DType::u64: code = CSPB_U64; break;
            default: break;
        }
        if (code < 0)
            throw std::invalid_argument("naga::cospan: " + who + ": '" + path + "' drives per-index extents by value and must "
                                        "have a 32- or 64-bit integer dtype");
        if (!src.produced) materialize(src);
        ensure_shape(src);
        if (offsets_mode ? src.rank != 1 : src.rank > 2)
            throw std::invalid_argument("naga::cospan: " + who + ": '" + path + "' drives per-index extents by value and must "
                                        "be rank 1" + std::string(offsets_mode ? " (N + 1 offsets)" : " [N] or rank 2 [N, k]"));
        const std::size_t count = src.shape[0];
        const std::size_t k = src.rank == 2 ? src.shape[1] : 1;
        if (offsets_mode && count == 0)
            throw std::invalid_argument("naga::cospan: " + who + ": '" + path + "' holds no offsets (it needs N + 1 >= 1 entries)");
        if (!offsets_mode && src.rank == 2 && k == 0)
            throw std::invalid_argument("naga::cospan: " + who + ": '" + path + "' has no column 0");
        if (!src.data) throw std::logic_error("naga::cospan: " + who + ": '" + path + "' has no data");
        const std::size_t n = offsets_mode ? count - 1 : count;
        if (!v.hook_column) v.hook_column = std::make_shared<Column>();
        Column& c = *v.hook_column;
        c.reserve(n, stream, wide);
        const std::size_t need = std::size_t(cspb_scan_workspace_bytes(std::int64_t(n)));
        if (need > scan_ws_bytes) {
            ++allocs;
            if (scan_ws) {
                cuda_check(cudaStreamSynchronize(stream), "a ragged hook's workspace");
                cudaFree(scan_ws);
                scan_ws = nullptr;
            }
            cuda_check(cudaMalloc(&scan_ws, need), "a ragged hook's workspace");
            scan_ws_bytes = need;
        }
        const int rc =
            wide ? cspb_build_column64(src.data, code, std::int64_t(count), std::int64_t(k), offsets_mode ? 1 : 0, c.ext,
                                       c.offs64, reinterpret_cast<std::uint64_t*>(c.tf_dev), scan_ws,
                                       std::int64_t(scan_ws_bytes), stream)
                 : cspb_build_column(src.data, code, std::int64_t(count), std::int64_t(k), offsets_mode ? 1 : 0, c.ext,
                                     c.offs, c.tf_dev, scan_ws, std::int64_t(scan_ws_bytes), stream);
        if (rc != 0) throw std::runtime_error("naga::cospan: " + who + ": building a ragged column: " + cspb_status_string(rc));
        cuda_check(cudaStreamSynchronize(stream), who);
        // [total, flag]: two u32, or two u64 whose second's low half holds the same flag bits
        const std::uint64_t total = wide ? reinterpret_cast<const std::uint64_t*>(c.tf)[0] : std::uint64_t(c.tf[0]);
        const std::uint32_t flag = wide ? c.tf[2] : c.tf[1];
        if (flag & CSPB_COLUMN_TIMEOUT)
            throw std::runtime_error("naga::cospan: " + who + ": '" + path + "': the device scan's bounded wait gave up "
                                     "(" + std::string(cspb_status_string(CSPB_ERR_TIMEOUT)) + ")");
        if ((flag & 1u) == 0 && (flag & 2u) != 0)
            throw std::invalid_argument(
                "naga::cospan: " + who + ": '" + path +
                (wide ? "' holds a block past 2^32 - 1 elements; a block's extent is a u32"
                      : "' holds a value or a total past 2^32 - 1; ragged totals with u32 offsets are limited to 2^32 - 1 "
                        "elements (cs::ragged::counts_from<std::uint64_t> takes u64 offsets)"));
        if (flag != 0)
            throw std::invalid_argument("naga::cospan: " + who + ": '" + path + "' holds " +
                                        std::string(offsets_mode ? "offsets that are negative, do not start at 0, or decrease"
                                                                 : "a negative value") + "; a size cannot be negative");
        c.n = n;
        c.total = total;
        ++c.version;
        c.has_upload = false;
        v.per = true;
        v.shape[0] = n;
        v.shape[1] = 0;
        v.total = total;
        v.host_counts.clear();
        v.column = v.hook_column;
        v.shape_known = true;
    }
    /// A ragged shape from host counts: uploaded into the variable's own column when they changed.
    void set_host_counts(Var& v, const std::vector<std::size_t>& counts, const std::string& who) {
        std::uint64_t total = 0;
        for (auto c : counts) {
            if (c > 0xFFFFFFFFull)
                throw std::invalid_argument("naga::cospan: " + who + ": a ragged block has " + std::to_string(c) +
                                            " elements; a block's extent is limited to 2^32 - 1");
            total += c;
        }
        // the host knows the total: past 2^32 - 1 the column takes u64 offsets by itself
        const bool wide = total > 0xFFFFFFFFull;
        if (!v.own_column) v.own_column = std::make_shared<Column>();
        Column& c = *v.own_column;
        if (!c.has_upload || c.uploaded != counts || c.wide != wide) {
            ++host_syncs;  // an upload from pageable memory: never part of a captured run
            c.reserve(counts.size(), stream, wide);
            c.staging.assign(2 * counts.size() + 1, 0u);
            c.staging64.assign(wide ? counts.size() + 1 : 0, 0u);
            std::uint64_t run = 0;
            for (std::size_t i = 0; i < counts.size(); ++i) {
                c.staging[i] = std::uint32_t(counts[i]);
                if (wide) c.staging64[i] = run;
                else c.staging[counts.size() + i] = std::uint32_t(run);
                run += counts[i];
            }
            if (wide) c.staging64[counts.size()] = run;
            else c.staging[2 * counts.size()] = std::uint32_t(run);
            // staging is pageable: each copy has consumed it when the call returns
            if (!counts.empty())
                cuda_check(cudaMemcpyAsync(c.ext, c.staging.data(), counts.size() * 4, cudaMemcpyHostToDevice, stream), who);
            if (wide)
                cuda_check(cudaMemcpyAsync(c.offs64, c.staging64.data(), (counts.size() + 1) * 8, cudaMemcpyHostToDevice,
                                           stream), who);
            else
                cuda_check(cudaMemcpyAsync(c.offs, c.staging.data() + counts.size(), (counts.size() + 1) * 4,
                                           cudaMemcpyHostToDevice, stream), who);
            c.uploaded = counts;
            c.has_upload = true;
            c.n = counts.size();
            c.total = total;
            ++c.version;
        }
        v.per = true;
        v.shape[0] = counts.size();
        v.shape[1] = 0;
        v.total = total;
        v.host_counts = counts;
        v.column = v.own_column;
        v.shape_known = true;
    }
    void ensure_shape(Var& v) {
        if (v.shape_known) return;
        if (!v.hook.empty()) {
            shape_from_hook(v);
            return;
        }
        if (v.declared_counts) {
            set_host_counts(v, *v.declared_counts, "'" + v.name + "'");
            return;
        }
        if (!v.spec.empty()) {
            bool all = true;
            for (int d = 0; d < v.rank; ++d) all = all && v.spec.known[d];
            if (all) {
                for (int d = 0; d < v.rank; ++d) v.shape[d] = v.spec.ext[d];
                v.shape_known = true;
                return;
            }
        }
        if (v.init && !v.init->shape && v.init->flat && v.rank == 1) {
            v.shape[0] = *v.init->flat;
            v.shape_known = true;
            return;
        }
        if (v.init && v.init->shape && int(v.init->shape->size()) == v.rank) {
            for (int d = 0; d < v.rank; ++d) v.shape[d] = (*v.init->shape)[d];
            v.shape_known = true;
            return;
        }
        throw std::invalid_argument("naga::cospan: the shape of '" + v.name + "' is not known (no declaration, hook, "
                                    "initializer or producer gives it)");
    }
    void allocate(Var& v) {
        const std::size_t b = std::max<std::size_t>(v.bytes(), 16);
        if (v.data && v.capacity >= b) return;
        ++allocs;
        if (v.data) {
            cuda_check(cudaStreamSynchronize(stream), "resize");
            cudaFree(v.data);
        }
        cuda_check(cudaMalloc(&v.data, b), "allocating '" + v.name + "'");
        // zeroed, so that a variable nothing has written yet (a hooked free input) reads the same on every run
        cuda_check(cudaMemsetAsync(v.data, 0, b, stream), "allocating '" + v.name + "'");
        v.capacity = b;
    }
    void materialize(Var& v) {
        ensure_shape(v);
        allocate(v);
        if (v.stale && v.init) {
            if (v.init->shape) {
                std::size_t n = 1;
                for (auto e : *v.init->shape) n *= e;
                if (n != v.elements())
                    throw std::invalid_argument("naga::cospan: the initializer of '" + v.name + "' has " + std::to_string(n) +
                                                " elements, the variable " + std::to_string(v.elements()));
            }
            InitTarget t{*this, v};
            v.init->run(t);
            v.stale = false;
            ++v.version;
            if (trace) std::fprintf(stderr, "[cospan] init var %d '%s' at %p (%zu elements)\n", v.id, v.name.c_str(), v.data,
                                    v.elements());
        }
    }

    // ---- names ----
    std::string resolve(System* s, const std::string& path) {
        auto a = s->aliases_.find(path);
        if (a != s->aliases_.end()) return resolve(s, a->second.target);
        auto t = tie_keys.find(s->path() + "/" + path);
        if (t != tie_keys.end()) return t->second;
        const auto dot = path.find('.');
        const std::string head = path.substr(0, dot);
        Node* c = s->child(head);
        if (!c)
            throw std::invalid_argument("naga::cospan: '" + (s->path().empty() ? std::string("<root>") : s->path()) +
                                        "' has no port or name '" + path + "'");
        if (dot == std::string::npos)
            throw std::invalid_argument("naga::cospan: '" + c->path() + "' is a subsystem, not a port");
        const std::string rest = path.substr(dot + 1);
        if (c->kind == Node::Kind::component) {
            auto* comp = static_cast<ComponentBase*>(c);
            if (!comp->port(rest))
                throw std::invalid_argument("naga::cospan: '" + comp->path() + "' has no port '" + rest + "'");
            return comp->path() + "." + rest;
        }
        return resolve(static_cast<System*>(c), rest);
    }
    Var& var_of_path(System* s, const std::string& path) {
        const std::string k = resolve(s, path);
        auto it = key_var.find(k);
        if (it == key_var.end()) throw std::logic_error("naga::cospan: '" + k + "' has no variable");
        return vars[it->second];
    }
    Var& var_of_port(ComponentBase* c, const std::string& port) { return vars[key_var.at(c->path() + "." + port)]; }

    // ---- running one component (a solo leaf, or a stage of a fused group) ----
    /// A variable whose declaration fixes zero elements needs no initializer (N = 0 stays valid).
    static bool declared_empty(const Var& v) {
        if (v.declared_counts) return v.declared_counts->empty();
        if (v.spec.empty() || v.spec.rank != v.rank) return false;
        for (int d = 0; d < v.rank; ++d)
            if (v.spec.known[d] && v.spec.ext[d] == 0) return true;
        return false;
    }
    /// Points a port's wrapper at its variable: a dense port gets the data and shape; a ragged one the data, N and
    /// the device column (or, on a dense rank-2 variable, the row length).
    void bind(ComponentBase* c, detail::PortRec& p, Var& v) {
        if (p.ragged) {
            if (v.per) p.bind_ragged(v.data, v.shape[0], v.column->offs, v.column->offs64, v.column->ext, 0);
            else p.bind_ragged(v.data, v.shape[0], nullptr, nullptr, nullptr, v.shape[1]);
            return;
        }
        if (v.per)
            throw std::logic_error("naga::cospan: '" + c->path() + "." + p.name + "' is ragged; declare it with RaggedInput / "
                                   "RaggedOutput (a dense Input / Output cannot see per-index extents)");
        p.bind(v.data, v.shape.data());
    }
    void prepare(ComponentBase* c) {
        c->rt_ = this;
        for (auto& p : c->ports_) {
            if (p.output) continue;
            Var& v = vars[p.var];
            if (!v.produced && !v.init && !v.data && v.hook.empty() && !declared_empty(v))
                throw std::invalid_argument("naga::cospan: the input '" + c->path() + "." + p.name + "' (variable '" +
                                            v.name + "') is never initialized");
            materialize(v);
            bind(c, p, v);
        }
        for (auto& p : c->ports_)
            if (p.output) {
                Var& v = vars[p.var];
                if (v.shape_from_prepare) v.shape_known = false;
            }
        c->prepare_forward();
        for (auto& p : c->ports_) {
            if (!p.output) continue;
            Var& v = vars[p.var];
            materialize(v);
            bind(c, p, v);
        }
    }
    void trace_ports(ComponentBase* c) {
        for (auto& p : c->ports_) {
            const Var& v = vars[p.var];
            std::fprintf(stderr, "[cospan]   %s %-8s var %3d %-28s %p shape", p.output ? "out" : "in ", p.name.c_str(), v.id,
                         v.name.c_str(), v.data);
            for (int d = 0; d < v.rank; ++d) std::fprintf(stderr, " %zu", v.shape[d]);
            if (v.per) std::fprintf(stderr, " (ragged, %llu elements)", (unsigned long long)v.total);
            std::fprintf(stderr, "\n");
        }
    }
    void run_component(ComponentBase* c) {
        prepare(c);
        if (trace) {
            std::fprintf(stderr, "[cospan] launch '%s'\n", c->path().c_str());
            trace_ports(c);
        }
        std::unique_ptr<LaunchDescription> d = c->define_forward();
        if (d) c->launch_solo(*this, *d);
    }
};

// ---- initializer kernels ----
template <class T>
__global__ void k_fill(T* p, std::size_t n, T v) {
    for (std::size_t i = std::size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += std::size_t(gridDim.x) * blockDim.x)
        p[i] = v;
}
template <class T>
inline void fill_var(Runtime& rt, Var& v, T value) {
    const std::size_t n = v.elements();
    if (n == 0) return;
    const unsigned blocks = unsigned(std::min<std::size_t>((n + 255) / 256, 65535));
    k_fill<T><<<blocks, 256, 0, rt.stream>>>(static_cast<T*>(v.data), n, value);
    cuda_check(cudaGetLastError(), "fill");
}
template <class V>
inline void fill_any(Runtime& rt, Var& v, V value) {
    switch (value_dtype(v.dtype)) {
        case DType::f32: fill_var<float>(rt, v, float(value)); break;
        case DType::f64: fill_var<double>(rt, v, double(value)); break;
        case DType::i32: fill_var<std::int32_t>(rt, v, std::int32_t(value)); break;
        case DType::u32: fill_var<std::uint32_t>(rt, v, std::uint32_t(value)); break;
        case DType::i64: fill_var<std::int64_t>(rt, v, std::int64_t(value)); break;
        case DType::u64: fill_var<std::uint64_t>(rt, v, std::uint64_t(value)); break;
        default: fill_var<std::uint8_t>(rt, v, std::uint8_t(value)); break;
    }
}

template <int R>
inline void set_range(sycl::range<R>& shape, sycl::range<R>& stride, const std::array<std::size_t, 4>& s) {
    std::size_t st = 1;
    for (int d = R - 1; d >= 0; --d) {
        shape[d] = s[d];
        stride[d] = st;
        st *= s[d];
    }
}

}  // namespace detail

// ---- initializers (init.hpp) ----------------------------------------------------------------------------------------
namespace init {
template <class T>
InitSpec fill(T value) {
    InitSpec s;
    s.scalar = double(value);
    s.run = [value](detail::InitTarget& t) { detail::fill_any(t.rt, t.var, value); };
    return s;
}
template <class T>
InitSpec fill(T value, const Shape& shape) {
    InitSpec s = fill(value);
    s.shape = shape.ext;
    return s;
}
inline InitSpec zero() { return fill(0); }
inline InitSpec zero(const Shape& shape) { return fill(0, shape); }
template <class T>
InitSpec from_host(std::vector<T> values) {
    // the flat form checks the element count only (the variable's own shape decides its rank)
    InitSpec s;
    auto data = std::make_shared<std::vector<T>>(std::move(values));
    const std::size_t n = data->size();
    s.run = [data, n](detail::InitTarget& t) {
        if (n != t.var.elements())
            throw std::invalid_argument("naga::cospan: init::from_host has " + std::to_string(n) + " values, '" + t.var.name +
                                        "' has " + std::to_string(t.var.elements()) + " elements");
        if (sizeof(T) != dtype_size(t.var.dtype))
            throw std::invalid_argument("naga::cospan: init::from_host for '" + t.var.name + "' has the wrong element type");
        ++t.rt.host_syncs;
        detail::cuda_check(cudaMemcpyAsync(t.var.data, data->data(), n * sizeof(T), cudaMemcpyHostToDevice, t.rt.stream),
                           "from_host");
        detail::cuda_check(cudaStreamSynchronize(t.rt.stream), "from_host");
    };
    s.flat = n;
    return s;
}
template <class T>
InitSpec from_host(std::vector<T> values, const Shape& shape) {
    if (shape.elements() != values.size())
        throw std::invalid_argument("naga::cospan: init::from_host has " + std::to_string(values.size()) +
                                    " values but its shape has " + std::to_string(shape.elements()) + " elements");
    InitSpec s = from_host(std::move(values));
    s.shape = shape.ext;
    return s;
}
template <DType DT, int R>
InitSpec custom(CustomFn<DT, R> fn) {
    InitSpec s;
    s.run = [fn = std::move(fn)](detail::InitTarget& t) {
        if (!dtype_compatible(t.var.dtype, DT) || t.var.rank != R)
            throw std::invalid_argument("naga::cospan: init::custom for '" + t.var.name +
                                        "' was declared with the wrong dtype or rank");
        Initializer<DT, R> w;
        w.data_ = static_cast<cpp_type_t<DT>*>(t.var.data);
        detail::set_range<R>(w.shape_, w.stride_, t.var.shape);
        sycl::device dev(t.rt.device);
        fn(*t.rt.uq, dev, std::vector<sycl::event>{}, w);
    };
    return s;
}
template <DType DT, int R>
InitSpec custom(CustomFn<DT, R> fn, const Shape& shape) {
    InitSpec s = custom<DT, R>(std::move(fn));
    s.shape = shape.ext;
    return s;
}
}  // namespace init

// ---- component pieces that need the runtime -------------------------------------------------------------------------
template <DType DT, int R>
sycl::range<R> ComponentBase::shape_of(const Input<DT, R>& w) const {
    for (const auto& p : ports_)
        if (p.wrapper == static_cast<const void*>(&w)) {
            detail::Var& v = rt_->vars[p.var];
            rt_->ensure_shape(v);
            if (v.per)
                throw std::logic_error("naga::cospan: '" + path() + "." + p.name + "' is ragged; declare it with RaggedInput");
            sycl::range<R> r;
            for (int d = 0; d < R; ++d) r[d] = v.shape[d];
            return r;
        }
    throw std::logic_error("naga::cospan: '" + path() + "': shape_of on a port it does not own");
}
template <DType DT, int R, class... E>
void ComponentBase::set_shape(Output<DT, R>& w, E... e) {
    static_assert(sizeof...(E) == R, "set_shape needs one extent per dimension");
    for (auto& p : ports_)
        if (p.wrapper == static_cast<const void*>(&w)) {
            detail::Var& v = rt_->vars[p.var];
            const std::array<std::size_t, 4> s{static_cast<std::size_t>(e)...};
            for (int d = 0; d < R; ++d) v.shape[d] = s[d];
            v.shape_known = true;
            v.shape_from_prepare = true;
            return;
        }
    throw std::logic_error("naga::cospan: '" + path() + "': set_shape on a port it does not own");
}

inline RaggedShape ComponentBase::ragged_shape_of(const void* w) const {
    for (const auto& p : ports_)
        if (p.wrapper == w) {
            detail::Var& v = rt_->vars[p.var];
            rt_->ensure_shape(v);
            RaggedShape r;
            r.n = v.shape[0];
            if (v.per) {
                r.total = v.total;
                r.counts = v.host_counts;
                r.column = v.column;
                r.column_version = v.column ? v.column->version : 0;
            } else {  // a dense variable reads as constant rows
                r.counts.assign(r.n, v.shape[1]);
                r.total = std::uint64_t(r.n) * v.shape[1];
            }
            return r;
        }
    throw std::logic_error("naga::cospan: '" + path() + "': shape_of on a port it does not own");
}
inline void ComponentBase::set_ragged_shape(const void* w, const RaggedShape& s) {
    for (auto& p : ports_)
        if (p.wrapper == w) {
            if (!p.output) throw std::logic_error("naga::cospan: '" + path() + "': set_shape on an input");
            detail::Var& v = rt_->vars[p.var];
            const std::string who = "set_shape('" + path() + "." + p.name + "')";
            if (v.declared_counts && !s.on_device() && *v.declared_counts != s.counts)
                throw std::invalid_argument("naga::cospan: " + who + ": the counts " + detail::list_of(s.counts) +
                                            " differ from the declared " + detail::list_of(*v.declared_counts));
            if (s.on_device()) {
                v.per = true;
                v.shape[0] = s.n;
                v.shape[1] = 0;
                v.total = s.total;
                v.host_counts = s.counts;
                v.column = std::const_pointer_cast<detail::Column>(s.column);
                v.shape_known = true;
            } else {
                if (s.counts.size() != s.n)
                    throw std::invalid_argument("naga::cospan: " + who + ": N is " + std::to_string(s.n) + " but " +
                                                std::to_string(s.counts.size()) + " counts were given");
                rt_->set_host_counts(v, s.counts, who);
            }
            v.shape_from_prepare = true;
            return;
        }
    throw std::logic_error("naga::cospan: '" + path() + "': set_shape on a port it does not own");
}

/// What a cs::dim::custom function reads (shape_hook.hpp:352-390 of the reference): shapes and values of variables
/// by path, in the namespace of the System that declared the hook.
class ShapeHookCtx {
public:
    struct Shape {
        int rank = 0;
        std::array<std::size_t, 4> extents{};
        bool ragged = false;
        std::uint64_t total = 0;
    };
    ShapeHookCtx(detail::Runtime& rt, System* sys, std::string target) : rt_(&rt), sys_(sys), target_(std::move(target)) {}
    Shape shape_of(std::string_view path) {
        detail::Var& v = rt_->var_of_path(sys_, std::string(path));
        if (!v.produced) rt_->materialize(v);
        rt_->ensure_shape(v);
        Shape r;
        r.rank = v.rank;
        r.extents = v.shape;
        r.ragged = v.per;
        r.total = v.per ? v.total : std::uint64_t(v.elements());
        return r;
    }
    std::size_t value_of(std::string_view path, std::size_t index) {
        detail::Var& v = rt_->var_of_path(sys_, std::string(path));
        return rt_->value_of(v, std::string(path), index, "the shape hook on '" + target_ + "'");
    }

private:
    detail::Runtime* rt_;
    System* sys_;
    std::string target_;
};
inline std::size_t detail::Runtime::custom_dim(Var& v, const dim::Custom& c) {
    ++host_syncs;  // a custom function may give another size on every run: such a model is never replayed
    ShapeHookCtx ctx(*this, v.hook_sys, v.hook_path.empty() ? v.name : v.hook_path);
    return c.fn(ctx);
}

namespace detail {
inline LocalLayout local_layout(const std::vector<std::size_t>& elem, const LaunchDescription& d, std::uint32_t base,
                                std::size_t& bytes, const std::string& who) {
    LocalLayout L;
    L.base = base;
    if (elem.size() != d.local.size())
        throw std::invalid_argument("naga::cospan: '" + who + "' declares " + std::to_string(elem.size()) +
                                    " local arrays but its launch describes " + std::to_string(d.local.size()));
    if (elem.size() > L.shapes.size()) throw std::invalid_argument("naga::cospan: '" + who + "': too many local arrays");
    std::size_t off = 0;
    for (std::size_t i = 0; i < elem.size(); ++i) {
        off = (off + 15) / 16 * 16;
        L.offsets[i] = off;
        L.shapes[i] = d.local[i];
        off += elem[i] * d.local[i][0] * d.local[i][1] * d.local[i][2];
    }
    bytes = (off + 15) / 16 * 16;
    return L;
}
inline void group_geometry(const LaunchDescription& d, int R, std::array<std::size_t, 3>& groups,
                           std::array<std::size_t, 3>& local, std::uint64_t& count, const std::string& who) {
    if (d.rank != R)
        throw std::invalid_argument("naga::cospan: '" + who + "': the launch range has rank " + std::to_string(d.rank) +
                                    ", the body " + std::to_string(R));
    count = 1;
    for (int k = 0; k < R; ++k) {
        local[k] = d.has_wg ? d.wg[k] : (k == R - 1 ? 128 : 1);
        if (local[k] == 0 || d.range[k] % local[k] != 0)
            throw std::invalid_argument("naga::cospan: '" + who + "': the launch range is not a multiple of the work-group");
        groups[k] = d.range[k] / local[k];
        count *= groups[k];
    }
}
}  // namespace detail

template <class X>
void Component<X>::launch_solo(detail::Runtime& rt, const LaunchDescription& d) {
    constexpr int R = detail::body_rank<X>;
    X* self = static_cast<X*>(this);
    if constexpr (!detail::is_group_body<X>) {
        if (d.rank != R) throw std::invalid_argument("naga::cospan: '" + path() + "': launch range of the wrong rank");
        sycl::range<R> r;
        std::uint64_t total = 1;
        for (int k = 0; k < R; ++k) {
            r[k] = d.range[k];
            total *= d.range[k];
        }
        if (total == 0) return;
        const unsigned blocks = unsigned(std::min<std::uint64_t>((total + 255) / 256, std::uint64_t(rt.sms) * 16));
        detail::k_index<X, R><<<blocks, 256, 0, rt.stream>>>(self->inputs, self->outputs, r, total);
    } else {
        std::array<std::size_t, 3> g3, l3;
        std::uint64_t count;
        detail::group_geometry(d, R, g3, l3, count, path());
        if (count == 0) return;
        sycl::range<R> groups, local;
        std::size_t threads = 1;
        for (int k = 0; k < R; ++k) {
            groups[k] = g3[k];
            local[k] = l3[k];
            threads *= l3[k];
        }
        std::size_t smem = 0;
        const detail::LocalLayout L = detail::local_layout(local_elem_sizes(), d, 0, smem, path());
        auto kern = detail::k_group<X, R>;
        if (smem > 48 * 1024)
            detail::cuda_check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)), path());
        const unsigned blocks = unsigned(std::min<std::uint64_t>(count, std::uint64_t(rt.sms) * 32));
        kern<<<blocks, unsigned(threads), smem, rt.stream>>>(self->inputs, self->outputs, groups, local, count, L);
    }
    detail::cuda_check(cudaGetLastError(), "launching '" + path() + "'");
}

namespace detail {
template <class List> struct fused_params_of;
template <class... Xs> struct fused_params_of<tlist<Xs...>> {
    using type = FusedParams<Xs...>;
    static constexpr std::size_t n = sizeof...(Xs);
    template <std::size_t... I>
    static void bind_io(type& p, const std::vector<ComponentBase*>& st, std::index_sequence<I...>) {
        ((std::get<I>(p.io) = std::make_pair(static_cast<Xs*>(st[I])->inputs, static_cast<Xs*>(st[I])->outputs)), ...);
    }
    static std::vector<std::vector<std::size_t>> elems() {
        return {[] {
            using LM = body_local_t<Xs>;
            if constexpr (std::is_void_v<LM>) return std::vector<std::size_t>{};
            else {
                auto a = local_arrays<LM>::elem_sizes();
                return std::vector<std::size_t>(a.begin(), a.end());
            }
        }()...};
    }
    static std::vector<int> ranks() { return {body_rank<Xs>...}; }
    static std::vector<bool> groups() { return {is_group_body<Xs>...}; }
    static const void* kernel() { return reinterpret_cast<const void*>(k_fused<Xs...>); }
};
}  // namespace detail

template <class Opts, class... Items>
void FusedGroup<Opts, Items...>::launch(detail::Runtime& rt) {
    using List = typename detail::stages_of_all<Items...>::type;
    using FP = detail::fused_params_of<List>;
    using P = typename FP::type;
    static_assert(FP::n <= detail::kMaxStages, "too many stages in one fused group");
    P p{};
    const auto elems = FP::elems();
    const auto ranks = FP::ranks();
    const auto kinds = FP::groups();
    const int nseg = int(segment_local_shared_.size());
    if (nseg > detail::kMaxSegments) throw std::invalid_argument("naga::cospan: '" + path() + "': too many segments");
    std::vector<std::size_t> seg_base(nseg, 0), seg_bytes(nseg, 0);
    std::size_t threads = 0;
    std::vector<std::unique_ptr<LaunchDescription>> descs(stages_.size());
    for (std::size_t i = 0; i < stages_.size(); ++i) {
        ComponentBase* c = stages_[i];
        rt.prepare(c);
        descs[i] = c->define_forward();
        if (!descs[i]) throw std::invalid_argument("naga::cospan: '" + c->path() + "' describes no launch");
    }
    // the work-group size: the group stages' (they must agree); 256 work-items when every stage is index-range
    for (std::size_t i = 0; i < stages_.size(); ++i) {
        if (!kinds[i]) continue;
        std::array<std::size_t, 3> g3{1, 1, 1}, l3{1, 1, 1};
        std::uint64_t cnt = 0;
        detail::group_geometry(*descs[i], ranks[i], g3, l3, cnt, stages_[i]->path());
        const std::size_t th = l3[0] * l3[1] * l3[2];
        if (threads == 0) threads = th;
        else if (threads != th)
            throw std::invalid_argument("naga::cospan: '" + path() + "': its stages have different work-group sizes");
    }
    if (threads == 0) threads = 256;
    for (std::size_t i = 0; i < stages_.size(); ++i) {
        ComponentBase* c = stages_[i];
        const LaunchDescription* d = descs[i].get();
        detail::StageGeom& g = p.st[i];
        const int s = stage_segment_[i];
        g.segment = std::uint32_t(s);
        if (!kinds[i]) {
            // an index-range stage: its range, flattened, in groups of `threads` work-items
            if (d->rank != ranks[i])
                throw std::invalid_argument("naga::cospan: '" + c->path() + "': launch range of the wrong rank");
            g.whole = 0;
            g.items = 1;
            for (int k = 0; k < ranks[i]; ++k) {
                g.groups[k] = d->range[k];
                g.items *= d->range[k];
            }
            g.count = (g.items + threads - 1) / threads;
            p.seg[s].count = std::max<std::uint64_t>(p.seg[s].count, g.count);
            continue;
        }
        g.whole = std::uint32_t(segment_whole_[s]);
        detail::group_geometry(*d, ranks[i], g.groups, g.local, g.count, c->path());
        std::size_t bytes = 0;
        const std::uint32_t base = segment_local_shared_[s] ? 0u : std::uint32_t(seg_bytes[s]);
        g.local_mem = detail::local_layout(elems[i], *d, base, bytes, c->path());
        seg_bytes[s] = segment_local_shared_[s] ? std::max(seg_bytes[s], bytes) : seg_bytes[s] + bytes;
        p.seg[s].count = std::max<std::uint64_t>(p.seg[s].count, g.count);
    }
    FP::bind_io(p, stages_, std::make_index_sequence<FP::n>{});
    p.nseg = std::uint32_t(nseg);
    p.ctrl = rt.ctrl;
    std::size_t smem = 0;
    for (auto b : seg_bytes) smem = std::max(smem, b);
    std::uint64_t most = 0;
    for (int s = 0; s < nseg; ++s) most = std::max(most, p.seg[s].count);
    if (most == 0 || threads == 0) return;
    const void* kern = FP::kernel();
    if (rt.trace) {
        std::fprintf(stderr, "[cospan] fused '%s': %d segments, %zu threads, %zu B local memory\n", path().c_str(), nseg,
                     threads, smem);
        for (std::size_t i = 0; i < stages_.size(); ++i) {
            const detail::StageGeom& g = p.st[i];
            std::fprintf(stderr, "[cospan]  stage '%s' segment %u %s count %llu groups %zu %zu %zu local %zu %zu %zu base %u\n",
                         stages_[i]->path().c_str(), g.segment, g.whole ? "whole" : "own", (unsigned long long)g.count,
                         g.groups[0], g.groups[1], g.groups[2], g.local[0], g.local[1], g.local[2], g.local_mem.base);
            rt.trace_ports(stages_[i]);
        }
    }
    if (smem > 48 * 1024)
        detail::cuda_check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)), path());
    int per_sm = 0;
    detail::cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, int(threads), smem), path());
    if (per_sm < 1) throw std::invalid_argument("naga::cospan: '" + path() + "': a work-group does not fit an SM");
    const unsigned grid = unsigned(std::min<std::uint64_t>(most, std::uint64_t(per_sm) * rt.sms));
    detail::cuda_check(cudaMemsetAsync(rt.ctrl + 1, 0, 8, rt.stream), "fused group barrier");
    void* args[] = {&p};
    if (nseg > 1)
        detail::cuda_check(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(unsigned(threads)), args, smem, rt.stream),
                           "launching '" + path() + "'");
    else
        detail::cuda_check(cudaLaunchKernel(kern, dim3(grid), dim3(unsigned(threads)), args, smem, rt.stream),
                           "launching '" + path() + "'");
    if (rt.trace) {
        const cudaError_t e = cudaStreamSynchronize(rt.stream);
        std::uint32_t st[3] = {0, 0, 0};
        cudaMemcpy(st, rt.ctrl, sizeof(st), cudaMemcpyDeviceToHost);
        std::fprintf(stderr, "[cospan] fused '%s': grid %u (%d per SM), sync %s, status %u barrier %u/%u\n", path().c_str(),
                     grid, per_sm, cudaGetErrorString(e), st[0], st[1], st[2]);
    }
}

// ---- host views (host_view.hpp:103-152) ------------------------------------------------------------------------------
template <DType DT, int R>
class HostView {
public:
    using value_type = cpp_type_t<DT>;
    explicit HostView(std::shared_ptr<detail::ViewState> s) : s_(std::move(s)) {}
    void sync() const {
        if (s_->ev) detail::cuda_check(cudaEventSynchronize(s_->ev), "view sync");
    }
    std::span<const value_type> span() const {
        return std::span<const value_type>(static_cast<const value_type*>(s_->host), s_->bytes / sizeof(value_type));
    }
    sycl::range<R> shape() const {
        sycl::range<R> r;
        for (int d = 0; d < R; ++d) r[d] = s_->shape[d];
        return r;
    }
    const value_type& operator[](std::size_t i) const { return span()[i]; }

private:
    std::shared_ptr<detail::ViewState> s_;
};

/// HostRagged<DT, 2>: a host view of a ragged variable (host_view.hpp:154-200 of the reference): the blocks end to
/// end, N, and the N + 1 block offsets. Also taken of a dense rank-2 variable, whose blocks are its rows.
template <DType DT, int R>
class HostRagged {
public:
    static_assert(R == 2, "naga::cospan: a ragged host view is rank 2");
    using value_type = cpp_type_t<value_dtype(DT)>;
    explicit HostRagged(std::shared_ptr<detail::ViewState> s) : s_(std::move(s)) {}
    void sync() const {
        if (s_->ev) detail::cuda_check(cudaEventSynchronize(s_->ev), "view sync");
    }
    std::size_t size() const { return s_->bytes / sizeof(value_type); }
    const value_type* data() const { return static_cast<const value_type*>(s_->host); }
    std::span<const value_type> span() const { return std::span<const value_type>(data(), size()); }
    const value_type& operator[](std::size_t f) const { return data()[f]; }
    /// N, the number of blocks.
    std::size_t n() const { return s_->n; }
    /// Block i is data()[offsets[i], offsets[i + 1]).
    std::vector<std::uint64_t> block_offsets() const {
        std::vector<std::uint64_t> o(s_->n + 1, 0);
        for (std::size_t i = 0; i <= s_->n; ++i) o[i] = s_->off(i);
        return o;
    }
    std::span<const value_type> block(std::size_t i) const {
        if (i >= s_->n) throw std::out_of_range("naga::cospan: HostRagged::block past the last block");
        const std::uint64_t a = s_->off(i);
        const std::uint64_t b = s_->off(i + 1);
        return std::span<const value_type>(data() + a, std::size_t(b - a));
    }

private:
    std::shared_ptr<detail::ViewState> s_;
};

// ---- the model --------------------------------------------------------------------------------------------------------
namespace detail {
void register_patterns(Runtime& rt);  // patterns.hpp
int verify_pattern(Runtime& rt, std::size_t pat);  // patterns.hpp
}

class Model {
public:
    explicit Model(std::unique_ptr<System> root) : root_(std::move(root)), rt_(std::make_unique<detail::Runtime>()) {}
    Model(Model&&) = default;
    Model& operator=(Model&&) = default;

    template <class T, class... A>
    void add_subsystem(const SubsystemDesc<T, A...>& d) { root_->add_subsystem(d); }
    template <class D, class = decltype(std::declval<const D&>().build())>
    void add_subsystem(const D& d) { root_->add_subsystem(d); }

    void setup() {
        if (setup_done_) return;
        root_->setup();
        setup_done_ = true;
    }
    void update_input(const std::string& path, InitSpec init) {
        finalize();
        detail::Var& v = rt_->var_of_path(root_.get(), path);
        if (v.produced)
            throw std::invalid_argument("naga::cospan: update_input('" + path + "'): the variable is an output of a component");
        v.init = std::move(init);
        v.stale = true;
        ++rt_->epoch;
        // the new initializer may bring another shape, unless the declaration fixes every dimension
        bool fixed = !v.spec.empty() && v.hook.empty();
        for (int d = 0; fixed && d < v.rank; ++d) fixed = v.spec.known[d];
        if (!fixed) v.shape_known = false;
    }
    /// One forward (model.hpp:471-480 of the reference): enqueues the leaves on the model's stream and returns.
    /// Steady runs replay a CUDA graph: once a run has made no host wait and no allocation (so every later run with
    /// the same inputs enqueues the same work), the next run is captured and later ones replay it with one launch,
    /// until update_input or a new host view. A capture that fails turns replay off for the model; the run is then
    /// done eagerly. NAGA_COSPAN_NO_GRAPH=1 turns replay off.
    void run() {
        finalize();
        auto& rt = *rt_;
        if (rt.graph_exec && rt.graph_epoch == rt.epoch) {
            detail::cuda_check(cudaGraphLaunch(rt.graph_exec, rt.stream), "replaying a forward");
            ++rt.graph_replays;
            for (auto& v : rt.views) push(*v);
            return;
        }
        if (rt.graph_allowed && rt.steady_epoch == rt.epoch && capture()) {
            for (auto& v : rt.views) push(*v);
            return;
        }
        const std::uint64_t syncs = rt.host_syncs, allocs = rt.allocs;
        run_leaves();
        rt.steady_epoch = rt.host_syncs == syncs && rt.allocs == allocs ? rt.epoch : ~0ull;
        for (auto& v : rt.views) push(*v);
    }
    /// How many forwards were captured into a graph, and how many replayed one.
    std::pair<std::uint64_t, std::uint64_t> graph_counts() const { return {rt_->graph_captures, rt_->graph_replays}; }

private:
    /// Captures one forward into a graph and launches it. False (nothing enqueued, replay turned off) when the capture
    /// failed or the forward waited on the host or allocated.
    bool capture() {
        auto& rt = *rt_;
        if (rt.graph_exec) {
            cudaGraphExecDestroy(rt.graph_exec);
            rt.graph_exec = nullptr;
        }
        const std::uint64_t syncs = rt.host_syncs, allocs = rt.allocs;
        if (cudaStreamBeginCapture(rt.stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
            cudaGetLastError();
            rt.graph_allowed = false;
            return false;
        }
        bool ok = true;
        try {
            run_leaves();
        } catch (const std::exception&) {
            ok = false;
        }
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(rt.stream, &g);
        ok = ok && e == cudaSuccess && g != nullptr && rt.host_syncs == syncs && rt.allocs == allocs;
        if (ok) ok = cudaGraphInstantiate(&rt.graph_exec, g, 0) == cudaSuccess;
        if (g) cudaGraphDestroy(g);
        if (!ok) {
            cudaGetLastError();
            if (rt.graph_exec) cudaGraphExecDestroy(rt.graph_exec);
            rt.graph_exec = nullptr;
            rt.graph_allowed = false;
            rt.steady_epoch = ~0ull;
            if (rt.trace) std::fprintf(stderr, "[cospan] capture failed: forwards run eagerly\n");
            run_leaves();  // the forward itself, eagerly
            return true;
        }
        rt.graph_epoch = rt.epoch;
        ++rt.graph_captures;
        detail::cuda_check(cudaGraphLaunch(rt.graph_exec, rt.stream), "launching a captured forward");
        return true;
    }
    void run_leaves() {
        auto& rt = *rt_;
        // shape hooks run once per forward, when their target's shape is first needed
        for (auto& v : rt.vars)
            if (!v.hook.empty()) v.shape_known = false;
        auto run_leaf = [&](std::size_t i) {
            Node* n = rt.leaves[i];
            if (n->kind == Node::Kind::component) rt.run_component(static_cast<ComponentBase*>(n));
            else static_cast<FusedGroupBase*>(n)->launch(rt);
        };
        for (std::size_t i = 0; i < rt.leaves.size(); ++i) {
            const int pat = rt.pattern_at.empty() ? -1 : rt.pattern_at[i];
            if (pat == -2) continue;
            if (pat >= 0) {
                const std::size_t hi = rt.pattern_hi[std::size_t(pat)];
                int& verified = rt.pattern_verified[std::size_t(pat)];
                if (verified == 0) {
                    // A run is recognised by its components' type names and wiring; before its kernel replaces the
                    // bodies, one forward runs both and compares what they write (never inside a graph capture: the
                    // comparison waits on the host)
                    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
                    cudaStreamIsCapturing(rt.stream, &cs);
                    for (std::size_t k = i; k <= hi; ++k) run_leaf(k);
                    if (cs == cudaStreamCaptureStatusNone) verified = detail::verify_pattern(rt, std::size_t(pat));
                    i = hi;
                    continue;
                }
                std::size_t next = i;
                if (verified > 0 && rt.pattern_runs[std::size_t(pat)](rt, next)) continue;
                // the fast path declined this run or disagreed with the bodies: the leaves it covers run their own
                for (std::size_t k = i; k <= hi; ++k) run_leaf(k);
                i = hi;
                continue;
            }
            run_leaf(i);
        }
    }

public:
    void wait() {
        detail::cuda_check(cudaStreamSynchronize(rt_->stream), "wait");
        std::uint32_t status = 0;
        detail::cuda_check(cudaMemcpy(&status, rt_->ctrl, 4, cudaMemcpyDeviceToHost), "status");
        if (status != 0) {
            cudaMemset(rt_->ctrl, 0, 256);
            throw std::runtime_error("naga::cospan: a device-side wait gave up (status " + std::to_string(status) + ")");
        }
    }
    template <DType DT, int R>
    HostView<DT, R> view_output(const std::string& path) { return dense_view<DT, R>("view_output", path); }
    template <DType DT, int R>
    HostView<DT, R> view_input(const std::string& path) { return dense_view<DT, R>("view_input", path); }
    /// A host view of a ragged variable (or of a dense rank-2 one, as rows), pushed after every run while it lives.
    template <DType DT, int R>
    HostRagged<DT, R> view_ragged_output(const std::string& path) { return ragged_view<DT, R>("view_ragged_output", path); }
    template <DType DT, int R>
    HostRagged<DT, R> view_ragged_input(const std::string& path) { return ragged_view<DT, R>("view_ragged_input", path); }
    System& root() { return *root_; }
    detail::Runtime& runtime() { return *rt_; }
    /// device bytes held by the model's variables (Model::memory_report's total)
    std::size_t memory_bytes() const {
        std::size_t b = 0;
        for (auto& v : rt_->vars) b += v.capacity;
        return b;
    }

private:
    std::unique_ptr<System> root_;
    std::unique_ptr<detail::Runtime> rt_;
    bool setup_done_ = false, finalized_ = false;

    template <DType DT, int R>
    HostView<DT, R> dense_view(const char* what, const std::string& path) {
        finalize();
        detail::Var& v = rt_->var_of_path(root_.get(), path);
        if (v.per || v.ragged_out)
            throw std::invalid_argument("naga::cospan: " + std::string(what) + "('" + path + "'): the variable is ragged; "
                                        "read it with view_ragged_" + std::string(what + 5));
        if (v.rank != R || !dtype_compatible(v.dtype, DT))
            throw std::invalid_argument("naga::cospan: " + std::string(what) + "('" + path + "'): wrong dtype or rank (the "
                                        "variable is " + std::string(dtype_name(v.dtype)) + " of rank " +
                                        std::to_string(v.rank) + ")");
        auto s = std::make_shared<detail::ViewState>();
        s->var = v.id;
        rt_->views.push_back(s);
        ++rt_->epoch;  // a viewed variable may change what the fast paths do
        push(*s);
        return HostView<DT, R>(s);
    }
    template <DType DT, int R>
    HostRagged<DT, R> ragged_view(const char* what, const std::string& path) {
        finalize();
        detail::Var& v = rt_->var_of_path(root_.get(), path);
        if (v.rank != R || R != 2 || !dtype_compatible(v.dtype, DT))
            throw std::invalid_argument("naga::cospan: " + std::string(what) + "('" + path + "'): wrong dtype or rank (the "
                                        "variable is " + std::string(dtype_name(v.dtype)) + " of rank " +
                                        std::to_string(v.rank) + ")");
        auto s = std::make_shared<detail::ViewState>();
        s->var = v.id;
        s->ragged = true;
        rt_->views.push_back(s);
        ++rt_->epoch;
        push(*s);
        return HostRagged<DT, R>(s);
    }
    void push(detail::ViewState& s) {
        detail::Var& v = rt_->vars[s.var];
        if (!v.data) return;
        const std::size_t b = v.bytes();
        if (b != s.bytes || !s.host) {
            if (s.host) cudaFreeHost(s.host);
            detail::cuda_check(cudaMallocHost(&s.host, std::max<std::size_t>(b, 16)), "host view");
            s.bytes = b;
        }
        s.shape = v.shape;
        s.per = v.per;
        s.n = v.shape[0];
        s.row = v.rank == 2 && !v.per ? v.shape[1] : 0;
        if (!s.ev) detail::cuda_check(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming), "view event");
        if (b) detail::cuda_check(cudaMemcpyAsync(s.host, v.data, b, cudaMemcpyDeviceToHost, rt_->stream), "view push");
        if (s.ragged && v.per) {
            const bool wide = v.column->wide;
            if (s.offs_cap < s.n + 1 || wide != (s.host_offs64 != nullptr)) {
                if (s.host_offs) cudaFreeHost(s.host_offs);
                if (s.host_offs64) cudaFreeHost(s.host_offs64);
                s.host_offs = nullptr;
                s.host_offs64 = nullptr;
                void** dst = wide ? reinterpret_cast<void**>(&s.host_offs64) : reinterpret_cast<void**>(&s.host_offs);
                detail::cuda_check(cudaMallocHost(dst, (s.n + 1) * (wide ? 8 : 4)), "host view");
                s.offs_cap = s.n + 1;
            }
            if (wide)
                detail::cuda_check(cudaMemcpyAsync(s.host_offs64, v.column->offs64, (s.n + 1) * 8, cudaMemcpyDeviceToHost,
                                                   rt_->stream), "view push");
            else
                detail::cuda_check(cudaMemcpyAsync(s.host_offs, v.column->offs, (s.n + 1) * 4, cudaMemcpyDeviceToHost,
                                                   rt_->stream), "view push");
        }
        detail::cuda_check(cudaEventRecord(s.ev, rt_->stream), "view event");
    }

    void finalize();
};

template <class T, class... Args>
Model create_model(Args&&... args) {
    auto root = std::make_unique<T>(std::forward<Args>(args)...);
    root->name = "";
    return Model(std::move(root));
}

}  // namespace naga::cospan
