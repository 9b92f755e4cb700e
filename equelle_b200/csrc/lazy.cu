// Deferred elementwise expressions (see eqg_internal.cuh).
//
// Generated Equelle code evaluates a formula one runtime call at a time; on
// collections of millions of faces each call of the one-kernel-per-operation
// path streams its operands and result through HBM (24 bytes per element for
// a binary operation).  Here value-only elementwise calls only record a node.
// When a value is needed, every pending node of that length (the handles the
// program still holds) is compiled into one straight-line program and
// evaluated by expr_kernel: one thread per element reads each leaf array
// once, keeps intermediates in shared memory, and writes the pending
// results.  Each node is computed with the expression the corresponding
// one-operation kernel uses (ops.cu), so results are bit-identical to the
// one-kernel-per-operation path.  Measured on the B200 (4096x4096 shallow
// water): 6.6x fewer launches, but each pass moves 24 bytes of shared
// memory per element and operation for its intermediates, so the step time
// is unchanged; the mode is therefore off by default (runtime parameter
// lazy=1).
#include "eqg_internal.cuh"

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <unordered_map>

namespace eqg {

namespace {

constexpr int kVmThreads = 128;
constexpr int kVmLanes = 4;     // elements per thread and decoded instruction
constexpr int kVmRegs = 24;     // shared-memory registers per element
constexpr int kVmLeaves = 24;
constexpr int kVmOuts = 24;
constexpr int kVmInstr = 160;
constexpr int kLazyMaxCost = 96;  // larger expressions materialize their operands first
// Recorded for fusion: an expression this large (counted as a tree) is
// evaluated when it is made, so that a program that never reads its values
// does not hold an unbounded DAG.  A time step of an explicit scheme is a few
// thousand.
constexpr double kFuseMaxCost = 1e7;
constexpr size_t kVmSmem = (size_t)kVmRegs * kVmLanes * kVmThreads * sizeof(double);

// One opcode per operation and operand form, so that an instruction is
// decoded once for kVmLanes elements.
enum VmOp : uint8_t {
    VM_LOAD, VM_LOADM, VM_CONST,
    VM_ADD, VM_SUB, VM_MUL, VM_DIV,          // x op y
    VM_ADDI, VM_SUBI, VM_MULI, VM_DIVI,      // x op imm
    VM_IADD, VM_ISUB, VM_IMUL, VM_IDIV,      // imm op x
    VM_NEG, VM_SQRT, VM_ABS,
    VM_CMP, VM_CMPI, VM_ICMP,                // comparison `sub`: x ? y, x ? imm, imm ? x
    VM_SEL, VM_LOGIC, VM_STORE, VM_STOREM
};

struct VmIns {
    uint8_t op, sub, dst, a, b, c, flag, pad;
    double imm;
};

struct VmProgram {
    int ninstr = 0, nleaves = 0, nouts = 0, pad = 0;
    const void* leaf[kVmLeaves] = {};
    void* out[kVmOuts] = {};
    VmIns code[kVmInstr] = {};
};

__device__ __forceinline__ bool vm_cmp(int op, double a, double b)
{
    switch (op) {
    case EQG_LT: return a < b;
    case EQG_LE: return a <= b;
    case EQG_GT: return a > b;
    case EQG_GE: return a >= b;
    case EQG_EQ: return a == b;
    default: return a != b;
    }
}

// Each block evaluates tiles of kVmLanes * blockDim elements; thread t owns
// elements base + t + k * blockDim (k < kVmLanes), so every load and store
// of an instruction is coalesced.  The program is uniform across the grid:
// decoding does not diverge.  Registers live in shared memory,
// [reg][lane][thread].  Each operation is the expression of the matching
// one-operation kernel (ops.cu: unary_kernel, select_kernel, ...).
__global__ void __launch_bounds__(kVmThreads) expr_kernel(const __grid_constant__ VmProgram p, int64_t n)
{
    extern __shared__ double smem[];
    const int t = threadIdx.x;
    const int T = blockDim.x;
    auto R = [&](int r, int k) -> double& { return smem[((size_t)r * kVmLanes + k) * T + t]; };
    for (int64_t base = (int64_t)blockIdx.x * kVmLanes * T; base < n; base += (int64_t)gridDim.x * kVmLanes * T) {
        for (int pc = 0; pc < p.ninstr; ++pc) {
            const VmIns q = p.code[pc];
#define VM_LANES(body)                                  \
    _Pragma("unroll") for (int k = 0; k < kVmLanes; ++k) \
    {                                                   \
        const int64_t e = base + t + (int64_t)k * T;    \
        (void)e;                                        \
        body;                                           \
    }
            switch (q.op) {
            case VM_LOAD: VM_LANES(R(q.dst, k) = e < n ? static_cast<const double*>(p.leaf[q.a])[e] : 0.0); break;
            case VM_LOADM:
                VM_LANES(R(q.dst, k) = (e < n && static_cast<const uint8_t*>(p.leaf[q.a])[e]) ? 1.0 : 0.0);
                break;
            case VM_CONST: VM_LANES(R(q.dst, k) = q.imm); break;
            case VM_ADD: VM_LANES(R(q.dst, k) = R(q.a, k) + R(q.b, k)); break;
            case VM_SUB: VM_LANES(R(q.dst, k) = R(q.a, k) - R(q.b, k)); break;
            case VM_MUL: VM_LANES(R(q.dst, k) = R(q.a, k) * R(q.b, k)); break;
            case VM_DIV: VM_LANES(R(q.dst, k) = R(q.a, k) / R(q.b, k)); break;
            case VM_ADDI: VM_LANES(R(q.dst, k) = R(q.a, k) + q.imm); break;
            case VM_SUBI: VM_LANES(R(q.dst, k) = R(q.a, k) - q.imm); break;
            case VM_MULI: VM_LANES(R(q.dst, k) = R(q.a, k) * q.imm); break;
            case VM_DIVI: VM_LANES(R(q.dst, k) = R(q.a, k) / q.imm); break;
            case VM_IADD: VM_LANES(R(q.dst, k) = q.imm + R(q.a, k)); break;
            case VM_ISUB: VM_LANES(R(q.dst, k) = q.imm - R(q.a, k)); break;
            case VM_IMUL: VM_LANES(R(q.dst, k) = q.imm * R(q.a, k)); break;
            case VM_IDIV: VM_LANES(R(q.dst, k) = q.imm / R(q.a, k)); break;
            case VM_NEG: VM_LANES(R(q.dst, k) = 0.0 - R(q.a, k)); break;  // V::Zero(n) - x
            case VM_SQRT: VM_LANES(R(q.dst, k) = sqrt(R(q.a, k))); break;
            case VM_ABS: VM_LANES(const double x = R(q.a, k); R(q.dst, k) = (x >= 0.0 ? 1.0 : -1.0) * x); break;
            case VM_CMP: VM_LANES(R(q.dst, k) = vm_cmp(q.sub, R(q.a, k), R(q.b, k)) ? 1.0 : 0.0); break;
            case VM_CMPI: VM_LANES(R(q.dst, k) = vm_cmp(q.sub, R(q.a, k), q.imm) ? 1.0 : 0.0); break;
            case VM_ICMP: VM_LANES(R(q.dst, k) = vm_cmp(q.sub, q.imm, R(q.a, k)) ? 1.0 : 0.0); break;
            case VM_SEL:  // iftrue * trueones + iffalse * falseones
                VM_LANES(const bool m = R(q.a, k) != 0.0; const double tt = m ? 1.0 : 0.0;
                         const double ff = m ? 0.0 : 1.0; R(q.dst, k) = R(q.b, k) * tt + R(q.c, k) * ff);
                break;
            case VM_LOGIC:
                VM_LANES(const bool x = R(q.a, k) != 0.0; const bool y = R(q.b, k) != 0.0;
                         R(q.dst, k) = (q.sub == EQG_AND ? (x && y) : q.sub == EQG_OR ? (x || y) : !x) ? 1.0 : 0.0);
                break;
            case VM_STORE:
                VM_LANES(if (e < n) static_cast<double*>(p.out[q.b])[e] = R(q.a, k));
                break;
            case VM_STOREM:
                VM_LANES(if (e < n) static_cast<uint8_t*>(p.out[q.b])[e] = R(q.a, k) != 0.0 ? 1 : 0);
                break;
            }
#undef VM_LANES
        }
    }
}

// A pending result: its node and the handle that owns it (a collection or
// a mask; neither for an operand evaluated on its own).
struct Root {
    LazyNode* node;
    eqg_coll* coll;
    eqg_mask* mask;
};

// Compiles the DAG under `roots` into `prog`: nodes in post-order (shared
// nodes and leaf arrays once), a register for each value from its
// definition to its last use, a store after each root.  False when a limit
// is exceeded.
bool compile(const std::vector<Root>& roots, VmProgram& prog)
{
    std::vector<LazyNode*> order;
    std::unordered_map<LazyNode*, int> index;      // node -> position in order
    std::unordered_map<const void*, int> leaf_of;  // leaf array -> node position
    std::vector<int> alias;                        // node position -> position holding its value
    std::vector<std::pair<LazyNode*, int>> stack;
    for (const Root& r : roots) {
        if (index.count(r.node)) continue;
        stack.push_back({r.node, 0});
        while (!stack.empty()) {
            auto& top = stack.back();
            LazyNode* v = top.first;
            LazyNode* kids[3] = {v->a.get(), v->b.get(), v->c.get()};
            if (top.second < 3) {
                LazyNode* k = kids[top.second++];
                if (k && !index.count(k)) stack.push_back({k, 0});
                continue;
            }
            stack.pop_back();
            if (index.count(v)) continue;
            const int pos = (int)order.size();
            index[v] = pos;
            order.push_back(v);
            int al = pos;
            if (v->op == LZ_LEAF) {
                auto it = leaf_of.find(v->leaf->ptr);
                if (it != leaf_of.end()) al = it->second;
                else leaf_of[v->leaf->ptr] = pos;
            }
            alias.push_back(al);
        }
    }
    if ((int)leaf_of.size() > kVmLeaves || (int)roots.size() > kVmOuts) return false;
    const int nn = (int)order.size();
    // last use of every value (by instruction position of its users; roots
    // are used by their store right after their definition)
    std::vector<int> last(nn, -1);
    auto use = [&](LazyNode* k, int at) {
        if (k) {
            const int v = alias[index[k]];
            last[v] = std::max(last[v], at);
        }
    };
    for (int i = 0; i < nn; ++i) {
        use(order[i]->a.get(), i);
        use(order[i]->b.get(), i);
        use(order[i]->c.get(), i);
    }
    for (const Root& r : roots) {
        const int v = alias[index[r.node]];
        last[v] = std::max(last[v], v);
    }
    std::vector<int> regof(nn, -1);
    std::vector<int> free_regs;
    for (int r = kVmRegs - 1; r >= 0; --r) free_regs.push_back(r);
    std::unordered_map<int, int> leaf_slot;
    std::vector<std::vector<int>> stores(nn);
    for (int k = 0; k < (int)roots.size(); ++k) stores[alias[index[roots[k].node]]].push_back(k);
    prog = VmProgram();
    auto emit = [&](const VmIns& q) {
        if (prog.ninstr >= kVmInstr) return false;
        prog.code[prog.ninstr++] = q;
        return true;
    };
    auto reg = [&](LazyNode* k) { return (uint8_t)regof[alias[index[k]]]; };
    for (int i = 0; i < nn; ++i) {
        if (alias[i] != i) continue;  // a repeated leaf array: the first one's register
        LazyNode* v = order[i];
        if (free_regs.empty()) return false;
        const int dst = free_regs.back();
        free_regs.pop_back();
        regof[i] = dst;
        VmIns q{};
        q.dst = (uint8_t)dst;
        q.sub = (uint8_t)v->sub;
        q.imm = v->s;
        q.flag = (uint8_t)v->scalar_left;
        switch (v->op) {
        case LZ_LEAF: {
            auto it = leaf_slot.find(i);
            int slot;
            if (it == leaf_slot.end()) {
                slot = prog.nleaves++;
                prog.leaf[slot] = v->leaf->ptr;
                leaf_slot[i] = slot;
            } else {
                slot = it->second;
            }
            q.op = v->mask ? VM_LOADM : VM_LOAD;
            q.a = (uint8_t)slot;
            break;
        }
        case LZ_CONST: q.op = VM_CONST; break;
        case LZ_BIN:
            q.op = (uint8_t)(VM_ADD + (v->sub - EQG_ADD));
            q.a = reg(v->a.get());
            q.b = reg(v->b.get());
            break;
        case LZ_BINS:
            q.op = (uint8_t)((v->scalar_left ? VM_IADD : VM_ADDI) + (v->sub - EQG_ADD));
            q.a = reg(v->a.get());
            break;
        case LZ_UNARY:
            q.op = v->sub == EQG_NEG ? VM_NEG : v->sub == EQG_SQRT ? VM_SQRT : VM_ABS;
            q.a = reg(v->a.get());
            break;
        case LZ_CMP: q.op = VM_CMP; q.a = reg(v->a.get()); q.b = reg(v->b.get()); break;
        case LZ_CMPS: q.op = v->scalar_left ? VM_ICMP : VM_CMPI; q.a = reg(v->a.get()); break;
        case LZ_SEL: q.op = VM_SEL; q.a = reg(v->a.get()); q.b = reg(v->b.get()); q.c = reg(v->c.get()); break;
        case LZ_LOGIC: q.op = VM_LOGIC; q.a = reg(v->a.get()); q.b = reg(v->b ? v->b.get() : v->a.get()); break;
        default: return false;  // operators are recorded only for fusion
        }
        if (!emit(q)) return false;
        for (int k : stores[i]) {
            VmIns st{};
            st.op = roots[k].node->mask ? VM_STOREM : VM_STORE;
            st.a = (uint8_t)dst;
            st.b = (uint8_t)k;
            if (!emit(st)) return false;
        }
        // free the registers whose values are not used after this point
        auto release = [&](LazyNode* k) {
            if (!k) return;
            const int p = alias[index[k]];
            if (last[p] == i && regof[p] >= 0) {
                free_regs.push_back(regof[p]);
                regof[p] = -2;  // released
            }
        };
        release(v->a.get());
        if (v->b != v->a) release(v->b.get());
        if (v->c != v->a && v->c != v->b) release(v->c.get());
        if (last[i] <= i && regof[i] >= 0) {  // used by nothing later (a root's store only)
            free_regs.push_back(regof[i]);
            regof[i] = -2;
        }
    }
    prog.nouts = (int)roots.size();
    return true;
}

// The node becomes a leaf over `values` (its owner and every expression
// that shares it read the array from now on).
void make_leaf(LazyNode* v, Buf values)
{
    v->op = LZ_LEAF;
    v->leaf = std::move(values);
    v->a.reset();
    v->b.reset();
    v->c.reset();
    v->m.reset();
    v->cost = 1;
}

void run_program(Core& c, const VmProgram& prog, int64_t n)
{
    if (n <= 0) return;
    static std::once_flag smem_set;
    std::call_once(smem_set, [] {
        EQG_CUDA(cudaFuncSetAttribute(expr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kVmSmem));
    });
    const int64_t tile = (int64_t)kVmLanes * kVmThreads;
    const int blocks = (int)std::min<int64_t>((n + tile - 1) / tile, 148 * 8);
    launch(c, "expr", [&] { expr_kernel<<<blocks, kVmThreads, kVmSmem, c.stream>>>(prog, n); });
    c.lazy_passes++;
}

// One node whose operands are evaluated, by the kernel its operation
// launches when it is not deferred (capi.cu).
void eval_node(Core& c, LazyNode* v)
{
    const int64_t n = v->n;
    Buf out = c.alloc((size_t)(n > 0 ? n : 1) * (v->mask ? 1 : 8));
    auto D = [](const LazyP& k) { return k->leaf->as<double>(); };
    auto M = [](const LazyP& k) { return k->leaf->as<uint8_t>(); };
    switch (v->op) {
    case LZ_CONST: k_fill(c, out->as<double>(), v->s, n); break;
    case LZ_BIN: k_binary(c, v->sub, D(v->a), D(v->b), out->as<double>(), n); break;
    case LZ_BINS: k_binary_scalar(c, v->sub, D(v->a), v->s, v->scalar_left, out->as<double>(), n); break;
    case LZ_UNARY: k_unary_value(c, v->sub, D(v->a), out->as<double>(), n); break;
    case LZ_CMP: k_compare(c, v->sub, D(v->a), D(v->b), out->as<uint8_t>(), n); break;
    case LZ_CMPS: k_compare_scalar(c, v->sub, D(v->a), v->s, v->scalar_left, out->as<uint8_t>(), n); break;
    case LZ_SEL: k_select_value(c, M(v->a), D(v->b), D(v->c), out->as<double>(), n); break;
    case LZ_LOGIC: k_mask_logic(c, v->sub, M(v->a), v->b ? M(v->b) : M(v->a), out->as<uint8_t>(), n); break;
    case LZ_OPMAT: opmat_apply_values(c, *v->m, D(v->a), out->as<double>()); break;
    default: fail(EQG_ERR_UNSUPPORTED, "unknown deferred operation");
    }
    make_leaf(v, out);
}

// Every pending node under `root`, operands first, one kernel per node.
void eval_per_node(Core& c, LazyNode* root)
{
    std::vector<std::pair<LazyNode*, int>> stack{{root, 0}};
    while (!stack.empty()) {
        const size_t top = stack.size() - 1;
        LazyNode* v = stack[top].first;
        if (v->op == LZ_LEAF) {
            stack.pop_back();
            continue;
        }
        const int k = stack[top].second;
        if (k < 3) {
            stack[top].second = k + 1;
            LazyNode* kid = k == 0 ? v->a.get() : k == 1 ? v->b.get() : v->c.get();
            if (kid && kid->op != LZ_LEAF) stack.push_back({kid, 0});
            continue;
        }
        stack.pop_back();
        eval_node(c, v);
    }
}

// The handle takes the values of its node, which has become a leaf.
void adopt(Core& c, const Root& r)
{
    if (r.coll) {
        r.coll->val = r.node->leaf;
        r.coll->lazy.reset();
        c.lazy_colls.erase(r.coll);
    } else if (r.mask) {
        r.mask->v = r.node->leaf;
        r.mask->lazy.reset();
        c.lazy_masks.erase(r.mask);
    }
}

// Evaluates `first` (pending) and every other pending handle of its length
// that fits into the same program.
void materialize(Core& c, Root first)
{
    if (!c.lazy_vm) {
        lazy_evaluate(c, first.node);
        adopt(c, first);
        return;
    }
    const int64_t n = first.node->n;
    std::vector<Root> roots{first};
    VmProgram prog;
    if (!compile(roots, prog)) {
        // too large on its own: evaluate its operands first
        for (LazyNode* k : {first.node->a.get(), first.node->b.get(), first.node->c.get()}) {
            if (!k || k->op == LZ_LEAF || k->op == LZ_CONST) continue;
            Buf vals = c.alloc((size_t)(n > 0 ? n : 1) * (k->mask ? 1 : 8));
            VmProgram sub;
            std::vector<Root> one{Root{k, nullptr, nullptr}};
            if (!compile(one, sub)) fail(EQG_ERR_UNSUPPORTED, "deferred expression too large");
            sub.out[0] = vals->ptr;
            run_program(c, sub, n);
            make_leaf(k, vals);
        }
        if (!compile(roots, prog)) fail(EQG_ERR_UNSUPPORTED, "deferred expression too large");
    }
    // add the other pending handles of this length while the program fits
    auto try_add = [&](Root r) {
        roots.push_back(r);
        VmProgram trial;
        if (compile(roots, trial)) {
            prog = trial;
            return;
        }
        roots.pop_back();
    };
    for (eqg_coll* x : c.lazy_colls)
        if (x != first.coll && x->lazy && x->lazy->n == n) try_add(Root{x->lazy.get(), x, nullptr});
    for (eqg_mask* m : c.lazy_masks)
        if (m != first.mask && m->lazy && m->lazy->n == n) try_add(Root{m->lazy.get(), nullptr, m});
    std::vector<Buf> outs(roots.size());
    for (size_t k = 0; k < roots.size(); ++k) {
        outs[k] = c.alloc((size_t)(n > 0 ? n : 1) * (roots[k].node->mask ? 1 : 8));
        prog.out[k] = outs[k]->ptr;
    }
    run_program(c, prog, n);
    if (c.verbose > 3)
        std::printf("        deferred evaluation: %lld elements, %d instructions, %d arrays read, %d written\n",
                    (long long)n, prog.ninstr, prog.nleaves, prog.nouts);
    for (size_t k = 0; k < roots.size(); ++k) {
        const Root& r = roots[k];
        make_leaf(r.node, outs[k]);
        if (r.coll) {
            r.coll->val = outs[k];
            r.coll->lazy.reset();
            c.lazy_colls.erase(r.coll);
        } else if (r.mask) {
            r.mask->v = outs[k];
            r.mask->lazy.reset();
            c.lazy_masks.erase(r.mask);
        }
    }
}

}  // namespace

void settle(Core& c, const eqg_coll* x)
{
    if (!x || !x->lazy) return;
    const Root r{x->lazy.get(), const_cast<eqg_coll*>(x), nullptr};
    // evaluated with another handle (a fused step's other results, or a
    // shared subexpression)
    if (r.node->op == LZ_LEAF) adopt(c, r);
    else materialize(c, r);
}

void settle(Core& c, const eqg_mask* m)
{
    if (!m || !m->lazy) return;
    const Root r{m->lazy.get(), nullptr, const_cast<eqg_mask*>(m)};
    if (r.node->op == LZ_LEAF) adopt(c, r);
    else materialize(c, r);
}

void lazy_make_leaf(LazyNode* v, Buf values) { make_leaf(v, std::move(values)); }

void lazy_evaluate(Core& c, LazyNode* v)
{
    if (v->op == LZ_LEAF) return;
    if (c.fuse && fused_materialize(c, v)) return;
    eval_per_node(c, v);
}

void settle_all(Core& c)
{
    while (!c.lazy_colls.empty()) settle(c, *c.lazy_colls.begin());
    while (!c.lazy_masks.empty()) settle(c, *c.lazy_masks.begin());
}

const double* coll_values(Core& c, const eqg_coll* x)
{
    settle(c, x);
    return x->val->as<double>();
}

const uint8_t* mask_values(Core& c, const eqg_mask* m)
{
    settle(c, m);
    return m->v->as<uint8_t>();
}

bool lazy_ok(const Core& c, const eqg_coll* x) { return c.lazy && !x->pat; }

LazyP lazy_node(const eqg_coll* x)
{
    if (x->lazy) return x->lazy;
    auto v = std::make_shared<LazyNode>();
    v->op = LZ_LEAF;
    v->n = x->n;
    v->leaf = x->val;
    return v;
}

LazyP lazy_node(const eqg_mask* m)
{
    if (m->lazy) return m->lazy;
    auto v = std::make_shared<LazyNode>();
    v->op = LZ_LEAF;
    v->mask = true;
    v->n = m->n;
    v->leaf = m->v;
    return v;
}

LazyP lazy_make(int op, int sub, int64_t n, bool mask, LazyP a, LazyP b, LazyP c, double s, int scalar_left)
{
    auto v = std::make_shared<LazyNode>();
    v->op = op;
    v->sub = sub;
    v->n = n;
    v->mask = mask;
    v->s = s;
    v->scalar_left = scalar_left;
    v->cost = 1 + (a ? a->cost : 0) + (b ? b->cost : 0) + (c ? c->cost : 0);
    v->a = std::move(a);
    v->b = std::move(b);
    v->c = std::move(c);
    return v;
}

LazyP lazy_opmat(const OpMatrixP& m, LazyP a)
{
    auto v = std::make_shared<LazyNode>();
    v->op = LZ_OPMAT;
    v->n = m->n_out;
    v->m = m;
    v->cost = 1 + a->cost;
    v->a = std::move(a);
    return v;
}

eqg_coll* lazy_coll(const CoreP& core, int64_t n, LazyP node)
{
    auto* x = new eqg_coll;
    x->core = core;
    x->n = n;
    x->lazy = std::move(node);
    core->lazy_colls.insert(x);
    if (x->lazy->cost > (core->lazy_vm ? kLazyMaxCost : kFuseMaxCost)) settle(*core, x);
    return x;
}

eqg_mask* lazy_mask(const CoreP& core, int64_t n, LazyP node)
{
    auto* m = new eqg_mask;
    m->core = core;
    m->n = n;
    m->lazy = std::move(node);
    core->lazy_masks.insert(m);
    if (m->lazy->cost > (core->lazy_vm ? kLazyMaxCost : kFuseMaxCost)) settle(*core, m);
    return m;
}

void lazy_forget(eqg_coll* x)
{
    if (x->lazy) x->core->lazy_colls.erase(x);
}

void lazy_forget(eqg_mask* m)
{
    if (m->lazy) m->core->lazy_masks.erase(m);
}

}  // namespace eqg
