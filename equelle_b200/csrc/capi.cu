// extern "C" entry points of libeqg.so (declared in include/eqg.h).
//
// Each call validates its arguments on the host, enqueues device work on the
// runtime's stream and returns handles to immutable device buffers.  Index
// maps for On/Extend, operator matrices and Jacobian sparsity patterns are
// cached by the ids of the sets/patterns involved, so the op sequence of a
// residual evaluation costs only numeric kernels from its second call on.
#include "eqg_internal.cuh"

#include <mutex>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

namespace eqg {
void build_grid(Core& c, eqg_set** builtin);
void build_grid_from_file(Core& c, const std::string& path, eqg_set** builtin);
void set_last_error(const std::string& msg);
}

using namespace eqg;

namespace {

thread_local std::string g_last_error;

// EQG_TRACE=1 in the environment prints every C-ABI call to stderr;
// EQG_HOST_PROFILE=1 prints, at exit, the host time spent in each entry
// point.
bool trace_enabled()
{
    static const bool on = std::getenv("EQG_TRACE") != nullptr;
    return on;
}

struct HostProfile {
    bool on = std::getenv("EQG_HOST_PROFILE") != nullptr;
    struct Entry {
        int64_t calls = 0, slow = 0;  // slow: over 1 ms
        double ms = 0.0, max_ms = 0.0;
    };
    std::map<std::string, Entry> calls;
    ~HostProfile()
    {
        if (!on) return;
        std::vector<std::pair<double, std::string>> v;
        for (auto& kv : calls) v.emplace_back(kv.second.ms, kv.first);
        std::sort(v.rbegin(), v.rend());
        for (auto& e : v) {
            const Entry& x = calls[e.second];
            std::fprintf(stderr, "[eqg host] %-28s %8lld calls %10.3f ms, %lld over 1 ms, max %.3f ms\n",
                         e.second.c_str(), (long long)x.calls, x.ms, (long long)x.slow, x.max_ms);
        }
    }
};
HostProfile g_host_profile;
std::mutex g_host_profile_mutex;  // runtimes may be driven from several threads

template <class F>
int guarded(const char* name, F&& f)
{
    const bool trace = trace_enabled();
    if (trace) {
        std::fprintf(stderr, "[eqg] %s\n", name);
        std::fflush(stderr);
    }
    const auto t0 = std::chrono::steady_clock::now();
    struct Timer {
        const char* name;
        std::chrono::steady_clock::time_point t0;
        ~Timer()
        {
            if (!g_host_profile.on) return;
            std::lock_guard<std::mutex> lock(g_host_profile_mutex);
            auto& e = g_host_profile.calls[name];
            const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            e.calls++;
            e.ms += ms;
            if (ms > 1.0) e.slow++;
            e.max_ms = std::max(e.max_ms, ms);
        }
    } timer{name, t0};
    try {
        f();
        if (trace) {
            std::fprintf(stderr, "[eqg] %s ok\n", name);
            std::fflush(stderr);
        }
        return EQG_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return EQG_ERR_MEMORY;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return EQG_ERR_ARG;
    }
}

void need(const void* p, const char* what)
{
    if (!p) fail(EQG_ERR_ARG, std::string("null handle: ") + what);
}

eqg_set* new_set(const CoreP& core, int entity, int64_t n, Buf idx)
{
    auto* s = new eqg_set;
    s->core = core;
    s->id = core->newId();
    s->entity = entity;
    s->n = n;
    s->idx = std::move(idx);
    return s;
}

eqg_coll* new_coll(const CoreP& core, int64_t n, Buf val, PatternP pat = nullptr, Buf jval = nullptr)
{
    auto* c = new eqg_coll;
    c->core = core;
    c->n = n;
    c->val = std::move(val);
    c->pat = std::move(pat);
    c->jval = std::move(jval);
    return c;
}

eqg_mask* new_mask(const CoreP& core, int64_t n, Buf v)
{
    auto* m = new eqg_mask;
    m->core = core;
    m->n = n;
    m->v = std::move(v);
    return m;
}

// Device error word: cleared, passed to kernels, then read back.
struct ErrWord {
    Core& c;
    Buf b;
    explicit ErrWord(Core& core) : c(core), b(core.allocN<int32_t>(1))
    {
        EQG_CUDA(cudaMemsetAsync(b->ptr, 0, 4, c.stream));
    }
    int32_t* ptr() { return b->as<int32_t>(); }
    int32_t read()
    {
        EQG_CUDA(cudaMemcpyAsync(c.pinned, b->ptr, 4, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        int32_t v;
        std::memcpy(&v, c.pinned, 4);
        return v;
    }
};

bool set_sorted(Core& c, eqg_set* s)
{
    if (s->sorted < 0) {
        if (s->identity || s->n <= 1) {
            s->sorted = 1;
        } else {
            Buf flag = c.allocN<int32_t>(1);
            k_fill_i32(c, flag->as<int32_t>(), 1, 1);
            k_is_strictly_sorted(c, s->idx->as<int32_t>(), s->n, flag->as<int32_t>());
            int32_t f = 0;
            EQG_CUDA(cudaMemcpyAsync(c.pinned, flag->ptr, 4, cudaMemcpyDeviceToHost, c.stream));
            c.sync();
            std::memcpy(&f, c.pinned, 4);
            s->sorted = f ? 1 : 0;
        }
    }
    return s->sorted == 1;
}

// Positions of `keys` in the sorted, duplicate-free `within`; error if any
// key is absent (subsetIndices, EquelleRuntimeCPU_impl.hpp:28-83).
Buf locate(Core& c, eqg_set* within, const eqg_set* keys)
{
    if (!set_sorted(c, within)) fail(EQG_ERR_ARG, "the superset of On/Extend is not sorted and duplicate free");
    Buf pos = c.allocN<int32_t>(keys->n > 0 ? keys->n : 1);
    ErrWord err(c);
    k_locate(c, within->identity ? nullptr : within->idx->as<int32_t>(), within->n, keys->idx->as<int32_t>(),
             pos->as<int32_t>(), keys->n, (int)within->n, err.ptr());
    if (err.read()) fail(EQG_ERR_ARG, "On/Extend: an element is not in the given superset");
    return pos;
}

enum MapKind { MAP_ON = 1, MAP_EXTEND = 2, MAP_SUBSET = 3, MAP_SUPERSET = 4 };

// Operator matrix of On(from -> to): row i selects row pos(to[i]) in from.
OpMatrixP on_matrix(Core& c, eqg_set* from, eqg_set* to)
{
    const auto key = std::make_tuple((int)MAP_ON, from->id, to->id, (int64_t)0);
    auto it = c.opmat_cache.find(key);
    if (it != c.opmat_cache.end()) return it->second;
    Buf pos = locate(c, from, to);
    OpMatrixP m = opmat_from_map(c, pos->as<int32_t>(), (int)to->n, (int)from->n, false);
    c.opmat_cache[key] = m;
    return m;
}

// Operator matrix of Extend(from -> to): row pos(from[i]) of the result is
// row i of the data, other rows are empty.
OpMatrixP extend_matrix(Core& c, eqg_set* from, eqg_set* to)
{
    const auto key = std::make_tuple((int)MAP_EXTEND, from->id, to->id, (int64_t)0);
    auto it = c.opmat_cache.find(key);
    if (it != c.opmat_cache.end()) return it->second;
    Buf pos = locate(c, to, from);
    Buf inv = c.allocN<int32_t>(to->n > 0 ? to->n : 1);
    k_fill_i32(c, inv->as<int32_t>(), -1, to->n);
    ErrWord err(c);
    k_scatter_inverse(c, pos->as<int32_t>(), from->n, inv->as<int32_t>(), err.ptr());
    if (err.read())
        fail(EQG_ERR_UNSUPPORTED, "Extend from a collection with repeated elements is not supported");
    OpMatrixP m = opmat_from_map(c, inv->as<int32_t>(), (int)to->n, (int)from->n, true);
    c.opmat_cache[key] = m;
    return m;
}

OpMatrixP span_matrix(Core& c, int kind, int64_t start, int64_t len, int64_t n_src, int64_t n_out)
{
    const int64_t code = (start << 32) ^ (len << 1) ^ n_out;
    const auto key = std::make_tuple(kind, (uint64_t)n_src, (uint64_t)start, code);
    auto it = c.opmat_cache.find(key);
    if (it != c.opmat_cache.end()) return it->second;
    std::vector<int32_t> ptr(n_out + 1, 0), src;
    std::vector<double> w;
    for (int64_t i = 0; i < n_out; ++i) {
        int64_t s = -1;
        if (kind == MAP_SUBSET) s = start + i;
        else if (i >= start && i < start + len) s = i - start;
        if (s >= 0) {
            src.push_back((int32_t)s);
            w.push_back(1.0);
        }
        ptr[i + 1] = (int32_t)src.size();
    }
    OpMatrixP m = opmat_from_host(c, (int)n_out, (int)n_src, ptr, src, w);
    c.opmat_cache[key] = m;
    return m;
}

// The Jacobian values of x with its deferred rules applied, stored in x in
// place of the deferred form (the collection's value does not change).
const double* materialized_jacobian(Core& c, const eqg_coll* x)
{
    if (x->jdef.n > 0) {
        eqg_coll* w = const_cast<eqg_coll*>(x);
        Buf jv = c.allocN<double>(x->pat->nnz > 0 ? x->pat->nnz : 1);
        jacobian_apply_deferred(c, x->jdef, *x->pat, x->jval->as<double>(), jv->as<double>());
        w->jval = jv;
        w->jdef = Deferred{};
        w->jkeep.clear();
    }
    return x->jval->as<double>();
}

// out takes from's Jacobian as it is: pattern, stored values, deferred rules.
eqg_coll* sharing_jacobian(eqg_coll* out, const eqg_coll* from)
{
    out->pat = from->pat;
    out->jval = from->jval;
    out->jdef = from->jdef;
    out->jkeep = from->jkeep;
    return out;
}

// out = M data: values by SpMV, Jacobian by the cached conservative product.
eqg_coll* apply_operator(const CoreP& cp, const OpMatrixP& mp, const eqg_coll* x)
{
    Core& c = *cp;
    const OpMatrix& m = *mp;
    if (x->n != m.n_src) fail(EQG_ERR_ARG, "operator applied to a collection of the wrong size");
    if (c.fuse && lazy_ok(c, x)) return lazy_coll(cp, m.n_out, lazy_opmat(mp, lazy_node(x)));
    Buf val = c.allocN<double>(m.n_out > 0 ? m.n_out : 1);
    opmat_apply_values(c, m, coll_values(c, x), val->as<double>());
    if (!x->pat) return new_coll(cp, m.n_out, val);
    PatternP p = pattern_spgemm(c, m, x->pat);
    // deferred rules on x's values go into the planned product; without a
    // plan, x is materialized first
    if (x->jdef.n > 0 && !spgemm_has_plan(*p)) materialized_jacobian(c, x);
    Buf jv = c.allocN<double>(p->nnz > 0 ? p->nnz : 1);
    spgemm_values(c, m, *x->pat, x->jval->as<double>(), *p, jv->as<double>(), &x->jdef);
    return new_coll(cp, m.n_out, val, p, jv);
}

// Rules that scale the rows of their one Jacobian operand (see DeferredRule).
bool deferrable_rule(int rule)
{
    switch (rule) {
    case JR_ADD:
    case JR_SUB:
    case JR_MUL:
    case JR_DIV:
    case JR_SCALE_CONST:
    case JR_DIV_BY_CONST:
    case JR_SQRT:
    case JR_SIGN:
    case JR_NEG:
    case JR_SELECT: return true;
    default: return false;
    }
}

// An elementwise rule's result: value `val`, Jacobian by the rule over the
// operands' Jacobians.  With one Jacobian operand the rule scales its rows:
// it is deferred (kept on the result, applied by the readers) instead of
// run, up to kMaxDeferred rules per Jacobian.  mask_keep: the mask buffer
// the rule reads, if any.
eqg_coll* jac_rule(const CoreP& cp, int64_t n, Buf val, JacArgs a, const eqg_coll* ca, const eqg_coll* cb,
                   Buf mask_keep = nullptr)
{
    Core& c = *cp;
    const PatternP pa = ca ? ca->pat : nullptr;
    const PatternP pb = cb ? cb->pat : nullptr;
    if (!pa && !pb) return new_coll(cp, n, val);
    if (pa && pb && pa->cols != pb->cols) fail(EQG_ERR_ARG, "Jacobians with different numbers of columns");
    if ((!pa || !pb) && deferrable_rule(a.rule) && c.jac_defer) {
        const eqg_coll* op = pa ? ca : cb;
        if (op->jdef.n >= kMaxDeferred) materialized_jacobian(c, op);
        eqg_coll* out = sharing_jacobian(new_coll(cp, n, val), op);
        DeferredRule& r = out->jdef.r[out->jdef.n++];
        r.rule = a.rule;
        r.side = pa ? 0 : 1;
        r.va = a.va;
        r.vb = a.vb;
        r.vout = a.vout;
        r.mask = a.mask;
        r.s = a.s;
        // the value arrays the rule reads stay alive with the result
        if (ca && ca->val) out->jkeep.push_back(ca->val);
        if (cb && cb->val) out->jkeep.push_back(cb->val);
        out->jkeep.push_back(val);
        if (mask_keep) out->jkeep.push_back(mask_keep);
        return out;
    }
    PatternP out = pa && pb ? pattern_union(c, pa, pb) : (pa ? pa : pb);
    a.pa = pa.get();
    a.ja = pa ? ca->jval->as<double>() : nullptr;
    a.da = pa ? ca->jdef : Deferred{};
    a.pb = pb.get();
    a.jb = pb ? cb->jval->as<double>() : nullptr;
    a.db = pb ? cb->jdef : Deferred{};
    Buf jv = c.allocN<double>(out->nnz > 0 ? out->nnz : 1);
    jacobian_elementwise(c, a, *out, jv->as<double>());
    return new_coll(cp, n, val, out, jv);
}

Buf upload(Core& c, const void* src, size_t bytes)
{
    Buf b = c.alloc(bytes);
    if (bytes) c.copy_to_device(b->ptr, src, bytes);
    return b;
}

void download(Core& c, void* dst, const void* src, size_t bytes)
{
    if (!bytes) return;
    c.copy_to_host(dst, src, bytes);
}

eqg_set* memo_set(const CoreP& cp, int op, const eqg_set* key_set)
{
    auto it = cp->derived_sets.find(std::make_tuple(op, key_set->id));
    if (it == cp->derived_sets.end()) return nullptr;
    eqg_set_retain(it->second);
    return it->second;
}

void remember_set(const CoreP& cp, int op, const eqg_set* key_set, eqg_set* s)
{
    eqg_set_retain(s);
    cp->derived_sets[std::make_tuple(op, key_set->id)] = s;
}

int mark(Core& c)
{
    Mark m;
    EQG_CUDA(cudaEventCreate(&m.ev));
    EQG_CUDA(cudaEventRecord(m.ev, c.stream));
    c.marks.push_back(m);
    return (int)c.marks.size() - 1;
}

}  // namespace

// Lets the library's other C entry points report through eqg_last_error().
void eqg::set_last_error(const std::string& msg) { g_last_error = msg; }

extern "C" {

const char* eqg_last_error(void) { return g_last_error.c_str(); }
const char* eqg_backend_name(void) { return "cuda-sm100a"; }

int eqg_runtime_create(int nparams, const char* const* keys, const char* const* values, eqg_runtime** out)
{
    return guarded(__func__, [&] {
        need(out, "out");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            cudaGetLastError();
            fail(EQG_ERR_DEVICE, "no CUDA device is visible; libeqg.so has no CPU implementation");
        }
        for (int i = 0; i < nparams; ++i)
            if (std::string(keys[i]) == "device") {
                const int dev = std::stoi(values[i]);
                if (dev < 0 || dev >= ndev) fail(EQG_ERR_ARG, "device index out of range");
                EQG_CUDA(cudaSetDevice(dev));
            }
        auto rt = std::make_unique<eqg_runtime>();
        rt->core = std::make_shared<Core>();
        Core& c = *rt->core;
        for (int i = 0; i < nparams; ++i) c.params[keys[i]] = values[i];
        c.dim = c.param_i("grid_dim", 2);
        c.nx = c.param_i("nx", 6);
        c.ny = c.param_i("ny", 1);
        c.nz = c.param_i("nz", 1);
        c.dx = c.param_d("dx", 1.0);
        c.dy = c.param_d("dy", 1.0);
        c.dz = c.param_d("dz", 1.0);
        c.verbose = c.param_i("verbose", 0);
        c.max_iter = c.param_i("max_iter", 10);
        c.abs_res_tol = c.param_d("abs_res_tol", 1e-6);
        c.timed_kernel = c.param_s("time_kernel", "");
        c.jac_concat = c.param_i("jac_concat", 1) != 0;
        c.jac_defer = c.param_i("jac_defer", 1) != 0;
        c.stencil_ops = c.param_i("stencil_ops", 1) != 0;
        c.span_share = c.param_i("span_share", 1) != 0;
        c.red_partials = c.allocN<double>((size_t)kRedBlocks * 4);
        c.red_counter = c.allocN<unsigned int>(1);
        if (c.params.count("grid_filename")) build_grid_from_file(c, c.params["grid_filename"], rt->builtin);
        else build_grid(c, rt->builtin);
        // deferred values: lazy=1 evaluates them with the expression kernel;
        // otherwise fuse=1 (the default where a fused step exists: 2D
        // Cartesian grids) records them for fused steps
        c.lazy_vm = c.param_i("lazy", 0) != 0;
        c.fuse = !c.lazy_vm && c.param_i("fuse", c.cartesian && c.dim == 2 ? 1 : 0) != 0;
        c.lazy = c.lazy_vm || c.fuse;
        for (auto* s : rt->builtin) {
            s->core = rt->core;
            s->id = c.newId();
        }
        *out = rt.release();
    });
}

void eqg_runtime_destroy(eqg_runtime* rt)
{
    if (!rt) return;
    try {
        for (auto*& s : rt->builtin) {
            eqg_set_release(s);
            s = nullptr;
        }
        for (auto& kv : rt->core->derived_sets) eqg_set_release(kv.second);
        rt->core->derived_sets.clear();
        rt->core->sync();
    } catch (...) {
    }
    delete rt;
}

int eqg_runtime_grid_info(const eqg_runtime* rt, eqg_grid_info* out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        const Core& c = *rt->core;
        out->dimensions = c.dim;
        out->nx = c.nx;
        out->ny = c.ny;
        out->nz = c.nz;
        out->dx = c.dx;
        out->dy = c.dy;
        out->dz = c.dz;
        out->number_of_cells = c.nc;
        out->number_of_faces = c.nf;
        out->number_of_interior_faces = c.nif;
    });
}

int eqg_runtime_synchronize(eqg_runtime* rt)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        rt->core->sync();
    });
}

int eqg_runtime_stats(const eqg_runtime* rt, eqg_stats* out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        const Core& c = *rt->core;
        out->kernel_launches = c.launches.load();
        out->newton_solves = c.newton_solves;
        out->newton_iterations = c.newton_iterations;
        out->linear_solves = c.solver.linear_solves;
        out->krylov_iterations = c.solver.krylov_iterations;
        out->refinement_sweeps = c.solver.refinement_sweeps;
        out->patterns_built = c.patterns_built;
        out->pattern_cache_hits = c.pattern_hits;
        out->device_bytes_in_use = c.bytes_in_use;
        out->device_bytes_peak = c.bytes_peak;
        out->last_linear_residual = c.solver.last_residual;
        out->last_matrix_rows = c.solver.last_rows;
        out->last_matrix_nnz = c.solver.last_nnz;
        out->last_block_size = c.solver.last_block_size;
        out->last_matrix_blocks = c.solver.last_blocks;
        out->timed_kernel_launches = (int64_t)c.timer_pairs.size();
        double ms = 0.0;
        for (auto& pr : c.timer_pairs) {
            float f = 0.f;
            EQG_CUDA(cudaEventSynchronize(pr.b));
            EQG_CUDA(cudaEventElapsedTime(&f, pr.a, pr.b));
            ms += f;
        }
        out->timed_kernel_ms = ms;
        out->residual_evaluations = c.residual_clock.count;
        out->residual_ms = c.residual_clock.total_ms();
        out->factor_ms = c.factor_clock.total_ms();
        out->krylov_ms = c.krylov_clock.total_ms();
        out->fused_evaluations = c.fused_evaluations;
    });
}

int eqg_runtime_reset_stats(eqg_runtime* rt)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        Core& c = *rt->core;
        c.launches = 0;
        c.newton_solves = c.newton_iterations = 0;
        c.solver = SolverStats{};
        c.patterns_built = c.pattern_hits = 0;
        c.fused_evaluations = 0;
        c.bytes_peak = c.bytes_in_use;
        for (auto& pr : c.timer_pairs) {
            cudaEventDestroy(pr.a);
            cudaEventDestroy(pr.b);
        }
        c.timer_pairs.clear();
        c.residual_clock.clear();
        c.factor_clock.clear();
        c.krylov_clock.clear();
    });
}

int eqg_runtime_kernel_profile(const eqg_runtime* rt, char* buf, int64_t len, int64_t* needed)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        const Core& c = *rt->core;
        // per kernel name: launches, ms, algorithmic bytes, launches that
        // stated their bytes
        struct Agg {
            int64_t launches = 0, with_bytes = 0;
            double ms = 0.0, bytes = 0.0;
        };
        std::map<std::string, Agg> agg;
        for (auto& pr : c.timer_pairs) {
            float f = 0.f;
            EQG_CUDA(cudaEventSynchronize(pr.b));
            EQG_CUDA(cudaEventElapsedTime(&f, pr.a, pr.b));
            auto& e = agg[pr.name];
            e.launches++;
            e.ms += f;
            if (pr.bytes >= 0) {
                e.bytes += pr.bytes;
                e.with_bytes++;
            }
        }
        std::string js = "{";
        for (auto& kv : agg) {
            if (js.size() > 1) js += ", ";
            char tmp[256];
            std::snprintf(tmp, sizeof(tmp), "\"%s\": [%lld, %.6f, %.0f, %lld]", kv.first.c_str(),
                          (long long)kv.second.launches, kv.second.ms, kv.second.bytes,
                          (long long)kv.second.with_bytes);
            js += tmp;
        }
        js += "}";
        *needed = (int64_t)js.size() + 1;
        if (buf && len > 0) {
            const size_t m = std::min((size_t)len - 1, js.size());
            std::memcpy(buf, js.data(), m);
            buf[m] = 0;
        }
    });
}

int eqg_runtime_mark(eqg_runtime* rt, int* mark_id)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        *mark_id = mark(*rt->core);
    });
}

int eqg_runtime_elapsed_ms(eqg_runtime* rt, int a, int b, double* ms)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        Core& c = *rt->core;
        if (a < 0 || b < 0 || a >= (int)c.marks.size() || b >= (int)c.marks.size())
            fail(EQG_ERR_ARG, "mark id out of range");
        EQG_CUDA(cudaEventSynchronize(c.marks[b].ev));
        float f = 0.f;
        EQG_CUDA(cudaEventElapsedTime(&f, c.marks[a].ev, c.marks[b].ev));
        *ms = f;
    });
}

int eqg_runtime_solve_marks(const eqg_runtime* rt, int64_t k, int* s, int* e)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        const Core& c = *rt->core;
        if (k < 0 || k >= (int64_t)c.solves.size()) fail(EQG_ERR_ARG, "solve index out of range");
        *s = c.solves[k].start_mark;
        *e = c.solves[k].end_mark;
    });
}

int eqg_runtime_solve_info(const eqg_runtime* rt, int64_t k, eqg_solve_info* out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        const Core& c = *rt->core;
        if (k < 0 || k >= (int64_t)c.solves.size()) fail(EQG_ERR_ARG, "solve index out of range");
        *out = c.solves[k];
    });
}

// ---- sets -------------------------------------------------------------------
int eqg_set_builtin(eqg_runtime* rt, int which, eqg_set** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        if (which < 0 || which > 5) fail(EQG_ERR_ARG, "unknown builtin set");
        eqg_set_retain(rt->builtin[which]);
        *out = rt->builtin[which];
    });
}

int eqg_set_from_host(eqg_runtime* rt, int entity, const int32_t* idx, int64_t n, eqg_set** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        Core& c = *rt->core;
        if (entity != EQG_CELLS && entity != EQG_FACES) fail(EQG_ERR_ARG, "bad entity kind");
        if (n < 0) fail(EQG_ERR_ARG, "negative size");
        const int64_t lim = entity == EQG_CELLS ? c.nc : c.nf;
        for (int64_t i = 0; i < n; ++i)
            if (idx[i] < -1 || idx[i] >= lim) fail(EQG_ERR_ARG, "entity index out of range");
        *out = new_set(rt->core, entity, n, upload(c, idx, (size_t)n * 4));
    });
}

int eqg_set_size(const eqg_set* s, int64_t* n)
{
    return guarded(__func__, [&] {
        need(s, "set");
        *n = s->n;
    });
}

int eqg_set_entity(const eqg_set* s, int* e)
{
    return guarded(__func__, [&] {
        need(s, "set");
        *e = s->entity;
    });
}

int eqg_set_to_host(const eqg_set* s, int32_t* out)
{
    return guarded(__func__, [&] {
        need(s, "set");
        download(*s->core, out, s->idx->ptr, (size_t)s->n * 4);
    });
}

void eqg_set_retain(eqg_set* s)
{
    if (s) s->refs++;
}

void eqg_set_release(eqg_set* s)
{
    if (s && --s->refs == 0) delete s;
}

static int neighbour(eqg_runtime* rt, const eqg_set* faces, int side, eqg_set** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(faces, "faces");
        const CoreP& cp = rt->core;
        if (faces->entity != EQG_FACES) fail(EQG_ERR_ARG, "firstCell/secondCell need a face collection");
        if (eqg_set* m = memo_set(cp, 10 + side, faces)) {
            *out = m;
            return;
        }
        Buf o = cp->allocN<int32_t>(faces->n > 0 ? faces->n : 1);
        ErrWord err(*cp);
        k_face_neighbour(*cp, faces->idx->as<int32_t>(), side, o->as<int32_t>(), faces->n, err.ptr());
        if (err.read()) fail(EQG_ERR_ARG, "firstCell/secondCell of an empty face");
        eqg_set* s = new_set(cp, EQG_CELLS, faces->n, o);
        remember_set(cp, 10 + side, faces, s);
        *out = s;
    });
}

int eqg_first_cell(eqg_runtime* rt, const eqg_set* f, eqg_set** out) { return neighbour(rt, f, 0, out); }
int eqg_second_cell(eqg_runtime* rt, const eqg_set* f, eqg_set** out) { return neighbour(rt, f, 1, out); }

int eqg_set_is_empty(eqg_runtime* rt, const eqg_set* s, eqg_mask** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(s, "set");
        Core& c = *rt->core;
        Buf m = c.allocN<uint8_t>(s->n > 0 ? s->n : 1);
        k_is_empty(c, s->idx->as<int32_t>(), m->as<uint8_t>(), s->n);
        *out = new_mask(rt->core, s->n, m);
    });
}

int eqg_set_on(eqg_runtime* rt, const eqg_set* data, const eqg_set* from, const eqg_set* to, eqg_set** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(data, "data");
        need(from, "from");
        need(to, "to");
        Core& c = *rt->core;
        if (data->n != from->n) fail(EQG_ERR_ARG, "On: data size differs from its set");
        if (from->entity != to->entity) fail(EQG_ERR_ARG, "On: sets of different entity kinds");
        OpMatrixP m = on_matrix(c, const_cast<eqg_set*>(from), const_cast<eqg_set*>(to));
        Buf o = c.allocN<int32_t>(to->n > 0 ? to->n : 1);
        k_gather_i32(c, data->idx->as<int32_t>(), m->src->as<int32_t>(), o->as<int32_t>(), to->n, -1);
        *out = new_set(rt->core, data->entity, to->n, o);
    });
}

int eqg_set_extend(eqg_runtime* rt, const eqg_set* data, const eqg_set* from, const eqg_set* to, eqg_set** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(data, "data");
        need(from, "from");
        need(to, "to");
        Core& c = *rt->core;
        if (data->n != from->n) fail(EQG_ERR_ARG, "Extend: data size differs from its set");
        if (from->entity != to->entity) fail(EQG_ERR_ARG, "Extend: sets of different entity kinds");
        Buf pos = locate(c, const_cast<eqg_set*>(to), from);
        Buf inv = c.allocN<int32_t>(to->n > 0 ? to->n : 1);
        k_fill_i32(c, inv->as<int32_t>(), -1, to->n);
        ErrWord err(c);
        k_scatter_inverse(c, pos->as<int32_t>(), from->n, inv->as<int32_t>(), err.ptr());
        if (err.read()) fail(EQG_ERR_UNSUPPORTED, "Extend from a collection with repeated elements is not supported");
        Buf o = c.allocN<int32_t>(to->n > 0 ? to->n : 1);
        k_gather_i32(c, data->idx->as<int32_t>(), inv->as<int32_t>(), o->as<int32_t>(), to->n, -1);
        *out = new_set(rt->core, data->entity, to->n, o);
    });
}

int eqg_set_select(eqg_runtime* rt, const eqg_mask* pred, const eqg_set* a, const eqg_set* b, eqg_set** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(pred, "predicate");
        need(a, "iftrue");
        need(b, "iffalse");
        Core& c = *rt->core;
        if (a->n != pred->n || b->n != pred->n) fail(EQG_ERR_ARG, "trinaryIf: size mismatch");
        if (a->entity != b->entity) fail(EQG_ERR_ARG, "trinaryIf: entity kinds differ");
        Buf o = c.allocN<int32_t>(pred->n > 0 ? pred->n : 1);
        k_set_select(c, mask_values(c, pred), a->idx->as<int32_t>(), b->idx->as<int32_t>(), o->as<int32_t>(),
                     pred->n);
        *out = new_set(rt->core, a->entity, pred->n, o);
    });
}

int eqg_set_check_subset(eqg_runtime* rt, const eqg_set* sub, const eqg_set* super, int* is_sorted, int* is_included)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(sub, "subset");
        need(super, "superset");
        Core& c = *rt->core;
        std::vector<int32_t> a(sub->n), b(super->n);
        download(c, a.data(), sub->idx->ptr, a.size() * 4);
        download(c, b.data(), super->idx->ptr, b.size() * 4);
        *is_sorted = std::is_sorted(a.begin(), a.end()) ? 1 : 0;
        *is_included = (*is_sorted && std::is_sorted(b.begin(), b.end()) &&
                        std::includes(b.begin(), b.end(), a.begin(), a.end()))
                           ? 1
                           : 0;
    });
}

// ---- masks --------------------------------------------------------------------
int eqg_mask_from_host(eqg_runtime* rt, const uint8_t* v, int64_t n, eqg_mask** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        if (n < 0) fail(EQG_ERR_ARG, "negative size");
        std::vector<uint8_t> norm(v, v + n);
        for (auto& x : norm) x = x ? 1 : 0;
        *out = new_mask(rt->core, n, upload(*rt->core, norm.data(), (size_t)n));
    });
}

int eqg_mask_size(const eqg_mask* m, int64_t* n)
{
    return guarded(__func__, [&] {
        need(m, "mask");
        *n = m->n;
    });
}

int eqg_mask_to_host(const eqg_mask* m, uint8_t* out)
{
    return guarded(__func__, [&] {
        need(m, "mask");
        mask_values(*m->core, m);
        download(*m->core, out, m->v->ptr, (size_t)m->n);
    });
}

void eqg_mask_retain(eqg_mask* m)
{
    if (m) m->refs++;
}

void eqg_mask_release(eqg_mask* m)
{
    if (m && --m->refs == 0) {
        lazy_forget(m);
        delete m;
    }
}

int eqg_mask_logic(eqg_runtime* rt, int op, const eqg_mask* a, const eqg_mask* b, eqg_mask** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "mask");
        if (op != EQG_NOT) {
            need(b, "mask");
            if (a->n != b->n) fail(EQG_ERR_ARG, "mask size mismatch");
        }
        if (op < EQG_AND || op > EQG_NOT) fail(EQG_ERR_ARG, "unknown mask operator");
        Core& c = *rt->core;
        Buf o = c.allocN<uint8_t>(a->n > 0 ? a->n : 1);
        if (c.lazy) {
            *out = lazy_mask(rt->core, a->n,
                             lazy_make(LZ_LOGIC, op, a->n, true, lazy_node(a), op == EQG_NOT ? nullptr : lazy_node(b)));
            return;
        }
        k_mask_logic(c, op, mask_values(c, a), op == EQG_NOT ? mask_values(c, a) : mask_values(c, b),
                     o->as<uint8_t>(), a->n);
        *out = new_mask(rt->core, a->n, o);
    });
}

// ---- scalar collections ------------------------------------------------------------
int eqg_coll_from_host(eqg_runtime* rt, const double* v, int64_t n, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        if (n < 0) fail(EQG_ERR_ARG, "negative size");
        *out = new_coll(rt->core, n, upload(*rt->core, v, (size_t)n * 8));
    });
}

int eqg_coll_constant(eqg_runtime* rt, double v, int64_t n, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        if (n < 0) fail(EQG_ERR_ARG, "negative size");
        Core& c = *rt->core;
        if (c.lazy) {
            *out = lazy_coll(rt->core, n, lazy_make(LZ_CONST, 0, n, false, nullptr, nullptr, nullptr, v));
            return;
        }
        Buf b = c.allocN<double>(n > 0 ? n : 1);
        k_fill(c, b->as<double>(), v, n);
        *out = new_coll(rt->core, n, b);
    });
}

int eqg_coll_size(const eqg_coll* c, int64_t* n)
{
    return guarded(__func__, [&] {
        need(c, "collection");
        *n = c->n;
    });
}

int eqg_output_begin(eqg_runtime* rt, const eqg_coll* x, int64_t* ticket)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(x, "collection");
        need(ticket, "ticket");
        Core& c = *rt->core;
        c.reap_outputs();
        const double* v = coll_values(c, x);
        Core::OutputCopy oc;
        oc.values = x->val;
        oc.n = x->n;
        oc.bytes = (size_t)(x->n > 0 ? x->n : 1) * sizeof(double);
        {
            std::lock_guard<std::mutex> lock(c.output_mutex);
            auto it = c.pinned_pool.lower_bound(oc.bytes);
            if (it != c.pinned_pool.end() && it->first <= 2 * oc.bytes) {
                oc.host = it->second;
                oc.bytes = it->first;
                c.pinned_pool.erase(it);
            }
        }
        if (!oc.host) EQG_CUDA(cudaMallocHost(&oc.host, oc.bytes));
        cudaEvent_t ready = nullptr;
        EQG_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        EQG_CUDA(cudaEventRecord(ready, c.stream));
        EQG_CUDA(cudaStreamWaitEvent(c.copy_stream, ready, 0));
        cudaEventDestroy(ready);
        if (x->n > 0)
            EQG_CUDA(cudaMemcpyAsync(oc.host, v, (size_t)x->n * sizeof(double), cudaMemcpyDeviceToHost,
                                     c.copy_stream));
        EQG_CUDA(cudaEventCreateWithFlags(&oc.done, cudaEventDisableTiming));
        EQG_CUDA(cudaEventRecord(oc.done, c.copy_stream));
        std::lock_guard<std::mutex> lock(c.output_mutex);
        *ticket = c.next_ticket++;
        c.output_copies.emplace(*ticket, std::move(oc));
    });
}

int eqg_output_wait(eqg_runtime* rt, int64_t ticket, const double** values, int64_t* n)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        Core& c = *rt->core;
        double* host = nullptr;
        cudaEvent_t done = nullptr;
        {
            std::lock_guard<std::mutex> lock(c.output_mutex);
            auto it = c.output_copies.find(ticket);
            if (it == c.output_copies.end()) fail(EQG_ERR_ARG, "unknown output ticket");
            host = it->second.host;
            done = it->second.done;
            *n = it->second.n;
        }
        EQG_CUDA(cudaEventSynchronize(done));
        *values = host;
    });
}

int eqg_output_release(eqg_runtime* rt, int64_t ticket)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        Core& c = *rt->core;
        std::lock_guard<std::mutex> lock(c.output_mutex);
        auto it = c.output_copies.find(ticket);
        if (it == c.output_copies.end()) fail(EQG_ERR_ARG, "unknown output ticket");
        Core::OutputCopy oc = std::move(it->second);
        c.output_copies.erase(it);
        cudaEventSynchronize(oc.done);
        cudaEventDestroy(oc.done);
        c.pinned_pool.emplace(oc.bytes, oc.host);
        oc.host = nullptr;
        c.output_released.push_back(std::move(oc));  // device buffer dropped by the runtime's thread
    });
}

int eqg_coll_evaluate(eqg_runtime* rt, const eqg_coll* x)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(x, "collection");
        settle(*rt->core, x);
    });
}

int eqg_coll_to_host(const eqg_coll* c, double* out)
{
    return guarded(__func__, [&] {
        need(c, "collection");
        coll_values(*c->core, c);
        download(*c->core, out, c->val->ptr, (size_t)c->n * 8);
    });
}

int eqg_coll_jacobian_info(const eqg_coll* c, int64_t* rows, int64_t* cols, int64_t* nnz)
{
    return guarded(__func__, [&] {
        need(c, "collection");
        if (!c->pat) {
            *rows = c->n;
            *cols = 0;
            *nnz = -1;
            return;
        }
        *rows = c->pat->rows;
        *cols = c->pat->cols;
        *nnz = c->pat->nnz;
    });
}

int eqg_coll_jacobian_to_host(const eqg_coll* c, int64_t* rowptr, int32_t* colind, double* vals)
{
    return guarded(__func__, [&] {
        need(c, "collection");
        if (!c->pat) fail(EQG_ERR_ARG, "collection has no Jacobian");
        Core& core = *c->core;
        const Pattern& p = *c->pat;
        if (rowptr) {
            std::vector<int32_t> rp(p.rows + 1);
            download(core, rp.data(), p.rowptr->ptr, rp.size() * 4);
            for (size_t i = 0; i < rp.size(); ++i) rowptr[i] = rp[i];
        }
        if (colind) download(core, colind, p.colind->ptr, (size_t)p.nnz * 4);
        if (vals) download(core, vals, materialized_jacobian(core, c), (size_t)p.nnz * 8);
    });
}

void eqg_coll_retain(eqg_coll* c)
{
    if (c) c->refs++;
}

void eqg_coll_release(eqg_coll* c)
{
    if (c && --c->refs == 0) {
        lazy_forget(c);
        delete c;
    }
}

int eqg_variable(eqg_runtime* rt, const eqg_coll* init, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(init, "collection");
        Core& c = *rt->core;
        if (init->n > INT32_MAX) fail(EQG_ERR_UNSUPPORTED, "collection too large");
        settle(c, init);
        *out = new_coll(rt->core, init->n, init->val, pattern_identity(c, (int)init->n), ones(c, init->n));
    });
}

int eqg_value_of(eqg_runtime* rt, const eqg_coll* x, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(x, "collection");
        settle(*rt->core, x);
        *out = new_coll(rt->core, x->n, x->val);
    });
}

int eqg_binary(eqg_runtime* rt, int op, const eqg_coll* a, const eqg_coll* b, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "lhs");
        need(b, "rhs");
        Core& c = *rt->core;
        if (a->n != b->n)
            fail(EQG_ERR_ARG, "size mismatch in binary operator: " + std::to_string(a->n) + " vs " + std::to_string(b->n));
        if (op < EQG_ADD || op > EQG_DIV) fail(EQG_ERR_ARG, "unknown binary operator");
        if (lazy_ok(c, a) && lazy_ok(c, b)) {
            *out = lazy_coll(rt->core, a->n, lazy_make(LZ_BIN, op, a->n, false, lazy_node(a), lazy_node(b)));
            return;
        }
        Buf val = c.allocN<double>(a->n > 0 ? a->n : 1);
        k_binary(c, op, coll_values(c, a), coll_values(c, b), val->as<double>(), a->n);
        // A sum with one Jacobian shares that Jacobian unchanged (Zero + J).
        if (op == EQG_ADD && (!a->pat || !b->pat)) {
            const eqg_coll* j = a->pat ? a : b;
            *out = sharing_jacobian(new_coll(rt->core, a->n, val), j);
            return;
        }
        if (op == EQG_SUB && !b->pat) {
            *out = sharing_jacobian(new_coll(rt->core, a->n, val), a);
            return;
        }
        JacArgs ja;
        ja.rule = op == EQG_ADD ? JR_ADD : op == EQG_SUB ? JR_SUB : op == EQG_MUL ? JR_MUL : JR_DIV;
        ja.va = a->val->as<double>();
        ja.vb = b->val->as<double>();
        *out = jac_rule(rt->core, a->n, val, ja, a, b);
    });
}

int eqg_binary_scalar(eqg_runtime* rt, int op, const eqg_coll* a, double s, int scalar_left, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "collection");
        Core& c = *rt->core;
        if (op < EQG_ADD || op > EQG_DIV) fail(EQG_ERR_ARG, "unknown binary operator");
        if (lazy_ok(c, a)) {
            *out = lazy_coll(rt->core, a->n,
                             lazy_make(LZ_BINS, op, a->n, false, lazy_node(a), nullptr, nullptr, s, scalar_left));
            return;
        }
        Buf val = c.allocN<double>(a->n > 0 ? a->n : 1);
        k_binary_scalar(c, op, coll_values(c, a), s, scalar_left, val->as<double>(), a->n);
        if (!a->pat) {
            *out = new_coll(rt->core, a->n, val);
            return;
        }
        JacArgs ja;
        const eqg_coll* left = nullptr;
        const eqg_coll* right = nullptr;
        switch (op) {
        case EQG_ADD:
            *out = sharing_jacobian(new_coll(rt->core, a->n, val), a);
            return;
        case EQG_SUB:
            if (!scalar_left) {
                *out = sharing_jacobian(new_coll(rt->core, a->n, val), a);
                return;
            }
            ja.rule = JR_NEG;
            left = a;
            break;
        case EQG_MUL:
            ja.rule = JR_SCALE_CONST;
            ja.s = s;
            left = a;
            break;
        case EQG_DIV:
            if (!scalar_left) {
                ja.rule = JR_DIV_BY_CONST;
                ja.s = s;
                left = a;
            } else {
                // V::Constant(s) / x: D3*(-D1*Jx), D1 = s, D3 = 1/(x*x)
                ja.rule = JR_DIV;
                ja.s = s;
                ja.vb = a->val->as<double>();
                right = a;
            }
            break;
        }
        *out = jac_rule(rt->core, a->n, val, ja, left, right);
    });
}

int eqg_unary(eqg_runtime* rt, int op, const eqg_coll* a, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "collection");
        Core& c = *rt->core;
        if (op < EQG_NEG || op > EQG_ABS) fail(EQG_ERR_ARG, "unknown unary operator");
        if (lazy_ok(c, a)) {
            *out = lazy_coll(rt->core, a->n, lazy_make(LZ_UNARY, op, a->n, false, lazy_node(a)));
            return;
        }
        Buf val = c.allocN<double>(a->n > 0 ? a->n : 1);
        k_unary_value(c, op, coll_values(c, a), val->as<double>(), a->n);
        JacArgs ja;
        ja.rule = op == EQG_NEG ? JR_NEG : op == EQG_SQRT ? JR_SQRT : JR_SIGN;
        ja.va = a->val->as<double>();
        ja.vout = val->as<double>();
        *out = jac_rule(rt->core, a->n, val, ja, a, nullptr);
    });
}

int eqg_compare(eqg_runtime* rt, int op, const eqg_coll* a, const eqg_coll* b, eqg_mask** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "lhs");
        need(b, "rhs");
        if (a->n != b->n) fail(EQG_ERR_ARG, "comparison size mismatch");
        if (op < EQG_LT || op > EQG_NE) fail(EQG_ERR_ARG, "unknown comparison");
        Core& c = *rt->core;
        if (c.lazy) {
            *out = lazy_mask(rt->core, a->n, lazy_make(LZ_CMP, op, a->n, true, lazy_node(a), lazy_node(b)));
            return;
        }
        Buf m = c.allocN<uint8_t>(a->n > 0 ? a->n : 1);
        k_compare(c, op, coll_values(c, a), coll_values(c, b), m->as<uint8_t>(), a->n);
        *out = new_mask(rt->core, a->n, m);
    });
}

int eqg_compare_scalar(eqg_runtime* rt, int op, const eqg_coll* a, double s, int scalar_left, eqg_mask** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "collection");
        if (op < EQG_LT || op > EQG_NE) fail(EQG_ERR_ARG, "unknown comparison");
        Core& c = *rt->core;
        if (c.lazy) {
            *out = lazy_mask(rt->core, a->n,
                             lazy_make(LZ_CMPS, op, a->n, true, lazy_node(a), nullptr, nullptr, s, scalar_left));
            return;
        }
        Buf m = c.allocN<uint8_t>(a->n > 0 ? a->n : 1);
        k_compare_scalar(c, op, coll_values(c, a), s, scalar_left, m->as<uint8_t>(), a->n);
        *out = new_mask(rt->core, a->n, m);
    });
}

int eqg_gradient(eqg_runtime* rt, const eqg_coll* a, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "collection");
        if (a->n != rt->core->nc) fail(EQG_ERR_ARG, "Gradient needs a collection on all cells");
        *out = apply_operator(rt->core, rt->core->grad, a);
    });
}

int eqg_neg_gradient(eqg_runtime* rt, const eqg_coll* a, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "collection");
        if (a->n != rt->core->nc) fail(EQG_ERR_ARG, "negGradient needs a collection on all cells");
        *out = apply_operator(rt->core, rt->core->ngrad, a);
    });
}

int eqg_interior_divergence(eqg_runtime* rt, const eqg_coll* a, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "collection");
        if (a->n != rt->core->nif) fail(EQG_ERR_ARG, "interiorDivergence needs a collection on interior faces");
        *out = apply_operator(rt->core, rt->core->div_interior, a);
    });
}

int eqg_divergence(eqg_runtime* rt, const eqg_coll* a, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "collection");
        const Core& c = *rt->core;
        if (a->n == c.nif) {
            *out = apply_operator(rt->core, c.div_interior, a);
            return;
        }
        if (a->n != c.nf) fail(EQG_ERR_ARG, "Divergence needs a collection on all or interior faces");
        *out = apply_operator(rt->core, c.div_full, a);
    });
}

int eqg_on(eqg_runtime* rt, const eqg_coll* data, const eqg_set* from, const eqg_set* to, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(data, "data");
        need(from, "from");
        need(to, "to");
        if (data->n != from->n) fail(EQG_ERR_ARG, "On: data size differs from its set");
        if (from->entity != to->entity) fail(EQG_ERR_ARG, "On: sets of different entity kinds");
        OpMatrixP m = on_matrix(*rt->core, const_cast<eqg_set*>(from), const_cast<eqg_set*>(to));
        *out = apply_operator(rt->core, m, data);
    });
}

int eqg_extend(eqg_runtime* rt, const eqg_coll* data, const eqg_set* from, const eqg_set* to, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(data, "data");
        need(from, "from");
        need(to, "to");
        if (data->n != from->n) fail(EQG_ERR_ARG, "Extend: data size differs from its set");
        if (from->entity != to->entity) fail(EQG_ERR_ARG, "Extend: sets of different entity kinds");
        OpMatrixP m = extend_matrix(*rt->core, const_cast<eqg_set*>(from), const_cast<eqg_set*>(to));
        *out = apply_operator(rt->core, m, data);
    });
}

int eqg_select(eqg_runtime* rt, const eqg_mask* pred, const eqg_coll* a, const eqg_coll* b, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(pred, "predicate");
        need(a, "iftrue");
        need(b, "iffalse");
        if (a->n != pred->n || b->n != pred->n) fail(EQG_ERR_ARG, "trinaryIf: size mismatch");
        Core& c = *rt->core;
        if (lazy_ok(c, a) && lazy_ok(c, b)) {
            *out = lazy_coll(rt->core, pred->n,
                             lazy_make(LZ_SEL, 0, pred->n, false, lazy_node(pred), lazy_node(a), lazy_node(b)));
            return;
        }
        Buf val = c.allocN<double>(pred->n > 0 ? pred->n : 1);
        const uint8_t* mv = mask_values(c, pred);
        k_select_value(c, mv, coll_values(c, a), coll_values(c, b), val->as<double>(), pred->n);
        JacArgs ja;
        ja.rule = JR_SELECT;
        ja.mask = mv;
        *out = jac_rule(rt->core, pred->n, val, ja, a, b, pred->v);
    });
}

int eqg_span_subset(eqg_runtime* rt, const eqg_coll* a, int64_t start, int64_t num, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "collection");
        if (start < 0 || num < 0 || start + num > a->n) fail(EQG_ERR_ARG, "span out of range");
        OpMatrixP m = span_matrix(*rt->core, MAP_SUBSET, start, num, a->n, num);
        *out = apply_operator(rt->core, m, a);
    });
}

int eqg_span_superset(eqg_runtime* rt, const eqg_coll* a, int64_t start, int64_t total, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "collection");
        if (start < 0 || start + a->n > total) fail(EQG_ERR_ARG, "span out of range");
        OpMatrixP m = span_matrix(*rt->core, MAP_SUPERSET, start, a->n, a->n, total);
        Core& c = *rt->core;
        if (!a->pat || !c.span_share) {
            *out = apply_operator(rt->core, m, a);
            return;
        }
        // The superset only inserts empty Jacobian rows: the product keeps
        // every entry, in order, with weight 1, so the result shares the
        // operand's Jacobian values (collections are immutable) under the
        // superset pattern.
        Buf val = c.allocN<double>(total > 0 ? total : 1);
        opmat_apply_values(c, *m, coll_values(c, a), val->as<double>());
        PatternP p = pattern_spgemm(c, *m, a->pat, false);
        if (p->nnz != a->pat->nnz) fail(EQG_ERR_DEVICE, "span superset changed the number of Jacobian entries");
        // deferred rules index the operand's rows, which the superset shifts
        materialized_jacobian(c, a);
        *out = new_coll(rt->core, total, val, p, a->jval);
    });
}

int eqg_reduce(eqg_runtime* rt, int op, const eqg_coll* a, double* out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "collection");
        if (op < EQG_MIN || op > EQG_PROD) fail(EQG_ERR_ARG, "unknown reduction");
        if (a->n == 0 && (op == EQG_MIN || op == EQG_MAX)) fail(EQG_ERR_ARG, "min/maxReduce of an empty collection");
        Core& c = *rt->core;
        if (c.fuse && a->lazy && a->lazy->op != LZ_LEAF && fused_reduce(c, op, a->lazy.get(), out)) return;
        *out = k_reduce(c, op, coll_values(c, a), a->n);
    });
}

int eqg_two_norm(eqg_runtime* rt, const eqg_coll* a, double* out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(a, "collection");
        *out = k_two_norm(*rt->core, coll_values(*rt->core, a), a->n);
    });
}

int eqg_measure(eqg_runtime* rt, const eqg_set* s, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(s, "set");
        Core& c = *rt->core;
        const double* src = s->entity == EQG_CELLS ? c.cell_volumes->as<double>() : c.face_areas->as<double>();
        Buf v = c.allocN<double>(s->n > 0 ? s->n : 1);
        ErrWord err(c);
        k_gather_f64(c, src, s->idx->as<int32_t>(), 0, 0, v->as<double>(), s->n, err.ptr());
        if (err.read()) fail(EQG_ERR_ARG, "norm of an empty entity");
        *out = new_coll(rt->core, s->n, v);
    });
}

int eqg_centroid(eqg_runtime* rt, const eqg_set* s, int comp, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(s, "set");
        Core& c = *rt->core;
        if (comp < 0 || comp >= c.dim) fail(EQG_ERR_ARG, "centroid component out of range");
        const bool cells = s->entity == EQG_CELLS;
        const double* src = cells ? c.cell_centroids->as<double>() : c.face_centroids->as<double>();
        Buf v = c.allocN<double>(s->n > 0 ? s->n : 1);
        ErrWord err(c);
        k_gather_f64(c, src, s->idx->as<int32_t>(), cells ? c.nc : c.nf, comp, v->as<double>(), s->n, err.ptr());
        if (err.read()) fail(EQG_ERR_ARG, "centroid of an empty entity");
        *out = new_coll(rt->core, s->n, v);
    });
}

int eqg_normal(eqg_runtime* rt, const eqg_set* s, int comp, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(s, "set");
        Core& c = *rt->core;
        if (s->entity != EQG_FACES) fail(EQG_ERR_ARG, "normal needs a face collection");
        if (comp < 0 || comp >= c.dim) fail(EQG_ERR_ARG, "normal component out of range");
        Buf v = c.allocN<double>(s->n > 0 ? s->n : 1);
        ErrWord err(c);
        k_normal(c, s->idx->as<int32_t>(), v->as<double>(), comp, s->n, err.ptr());
        if (err.read()) fail(EQG_ERR_ARG, "normal of an empty face");
        *out = new_coll(rt->core, s->n, v);
    });
}

int eqg_solve_for_update(eqg_runtime* rt, const eqg_coll* residual, eqg_coll** du)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(residual, "residual");
        Core& c = *rt->core;
        if (!residual->pat) fail(EQG_ERR_ARG, "solveForUpdate: residual has no Jacobian");
        if (residual->pat->rows != residual->pat->cols) fail(EQG_ERR_ARG, "solveForUpdate: Jacobian is not square");
        Buf x = c.allocN<double>(residual->n > 0 ? residual->n : 1);
        SolveResult r = linear_solve(c, residual->pat, materialized_jacobian(c, residual), coll_values(c, residual),
                                     x->as<double>());
        c.solver.linear_solves++;
        c.solver.krylov_iterations += r.iterations;
        c.solver.refinement_sweeps += r.sweeps;
        c.solver.last_residual = r.rel_residual;
        c.solver.last_rows = residual->pat->rows;
        c.solver.last_nnz = residual->pat->nnz;
        c.solver.last_block_size = r.block_size;
        c.solver.last_blocks = r.blocks;
        if (c.verbose > 2)
            std::printf("        solveForUpdate: BiCGStab+ILU0 %d iterations (%d sweeps), rel. residual %g\n",
                        r.iterations, r.sweeps, r.rel_residual);
        if (!r.converged) fail(EQG_ERR_SOLVER, "Linear solver convergence failure.");
        *du = new_coll(rt->core, residual->n, x);
    });
}

int eqg_newton_solve(eqg_runtime* rt, eqg_residual_fn fn, void* user, const eqg_coll* u0, eqg_coll** out)
{
    return guarded(__func__, [&] {
        need(rt, "runtime");
        need(u0, "initial guess");
        if (!fn) fail(EQG_ERR_ARG, "null residual function");
        Core& c = *rt->core;
        // values deferred before the solve are evaluated now; inside it
        // every operation runs when it is called (the residual callbacks)
        settle_all(c);
        struct NoDeferral {
            Core& c;
            bool lazy, fuse;
            ~NoDeferral()
            {
                c.lazy = lazy;
                c.fuse = fuse;
            }
        } no_deferral{c, c.lazy, c.fuse};
        c.lazy = c.fuse = false;
        // flush_l2=<MB>: that many MB written before the solve's start mark,
        // so that a solve timed between its own marks finds none of its data
        // in L2 (for working sets smaller than L2)
        const int flush_mb = c.param_i("flush_l2", 0);
        if (flush_mb > 0) {
            const size_t nbytes = (size_t)flush_mb << 20;
            if (!c.flush_buf || c.flush_buf->bytes < nbytes) c.flush_buf = c.alloc(nbytes);
            EQG_CUDA(cudaMemsetAsync(c.flush_buf->ptr, 0, nbytes, c.stream));
        }
        const int m0 = mark(c);
        c.newton_solves++;
        const int64_t krylov0 = c.solver.krylov_iterations;
        const int64_t launches0 = c.launches.load();
        const size_t rp0 = c.residual_clock.pairs.size(), fp0 = c.factor_clock.pairs.size(),
                     kp0 = c.krylov_clock.pairs.size();
        struct Ref {
            eqg_coll* p = nullptr;
            ~Ref() { eqg_coll_release(p); }
            void reset(eqg_coll* q)
            {
                eqg_coll_release(p);
                p = q;
            }
        } u, res;
        eqg_coll* tmp = nullptr;
        if (eqg_variable(rt, u0, &tmp) != EQG_OK) fail(EQG_ERR_ARG, g_last_error);
        u.reset(tmp);
        tmp = nullptr;
        auto evaluate = [&](eqg_coll* uu, eqg_coll** r) {
            c.residual_clock.start(c.stream);
            const int st = fn(user, uu, r);
            c.residual_clock.stop(c.stream);
            return st;
        };
        if (evaluate(u.p, &tmp) != 0 || !tmp) fail(EQG_ERR_CALLBACK, "residual callback failed");
        res.reset(tmp);
        if (res.p->n != u.p->n) fail(EQG_ERR_ARG, "newtonSolve: residual and unknown differ in size");
        double norm = k_two_norm(c, coll_values(c, res.p), res.p->n);
        int iter = 0;
        if (c.verbose > 1)
            std::printf("    newtonSolve: iter = %d (max = %d), norm(residual) = %g (tol = %g)\n", iter, c.max_iter,
                        norm, c.abs_res_tol);
        while (norm > c.abs_res_tol && iter < c.max_iter) {
            eqg_coll* du = nullptr;
            const int st = eqg_solve_for_update(rt, res.p, &du);
            if (st != EQG_OK) fail(st, g_last_error);
            eqg_coll* un = nullptr;
            const int st2 = eqg_binary(rt, EQG_SUB, u.p, du, &un);
            eqg_coll_release(du);
            if (st2 != EQG_OK) fail(st2, g_last_error);
            u.reset(un);
            res.reset(nullptr);
            tmp = nullptr;
            if (evaluate(u.p, &tmp) != 0 || !tmp) fail(EQG_ERR_CALLBACK, "residual callback failed");
            res.reset(tmp);
            norm = k_two_norm(c, coll_values(c, res.p), res.p->n);
            ++iter;
            c.newton_iterations++;
            if (c.verbose > 1)
                std::printf("    newtonSolve: iter = %d (max = %d), norm(residual) = %g (tol = %g)\n", iter,
                            c.max_iter, norm, c.abs_res_tol);
        }
        if (c.verbose > 0) {
            if (norm > c.abs_res_tol) std::printf("Newton solver failed to converge in %d iterations\n", c.max_iter);
            else std::printf("Newton solver converged in %d iterations\n", iter);
        }
        settle(c, u.p);
        *out = new_coll(rt->core, u.p->n, u.p->val);
        eqg_solve_info info{};
        info.start_mark = m0;
        info.newton_iterations = iter;
        info.converged = norm <= c.abs_res_tol ? 1 : 0;
        info.krylov_iterations = c.solver.krylov_iterations - krylov0;
        info.kernel_launches = c.launches.load() - launches0;
        info.residual_ms = c.residual_clock.ms_from(rp0);
        info.factor_ms = c.factor_clock.ms_from(fp0);
        info.krylov_ms = c.krylov_clock.ms_from(kp0);
        info.end_mark = mark(c);
        c.solves.push_back(info);
    });
}

}  // extern "C"
