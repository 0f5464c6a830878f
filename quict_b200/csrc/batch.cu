// Persistent batch kernel: energies and adjoint gradients of many independent
// problems -- circuits of different qubit counts, observables and parameters
// -- in ONE kernel launch.
//
// Every instance i owns a pair vector of 2^(n_i + 1) amplitudes in one state
// pool (psi in the first half, lam in the second) and runs a chain of stages:
//
//   forward passes   register passes over psi; the first reads |0...0>
//   HAM              lam = H psi and FP64 partials of <psi|lam>
//   backward passes  adjoint pair passes over (psi, lam) with EXPECT ops
//   FIN              energy = sum of the HAM partials; gradient = W Im(sum of
//                    the EXPECT partials per slot), W the parameter weights
//
// A stage is split into work items (a range of tiles or amplitudes).  The
// host orders all items of all instances in one list: stage r of every
// instance comes before stage r + 1 of any, large instances first within a
// round.  Persistent CTAs take items in list order from one atomic counter.
// An item starts once its instance's done-counter reaches the number of that
// instance's items in earlier stages; those items precede it in the list, so
// the CTAs that took them are already running and no wait can deadlock.  Each
// wait is bounded (`timeout_ns` of global time): past it the kernel records
// the item in the control words and every CTA stops at its next wait.
//
// The reference has neither gradients nor batching (SURVEY: the quict_ml
// package is absent); the per-pass work is the register-tile pass of
// regtile.cuh, the observable term rule is qs_apply_pauli_sum's (observe.cu).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "batch.cuh"
#include "common.cuh"
#include "jit.h"
#include "regtile.cuh"

namespace qs {
namespace {

template <typename V, int R>
__global__ void __launch_bounds__(256, 1)
k_batch(const unsigned char* __restrict__ blob, V* __restrict__ states, const V* __restrict__ mats,
        double* __restrict__ parts, double* __restrict__ energies, double* __restrict__ grads,
        unsigned long long* __restrict__ ctrl, uint64_t timeout_ns) {
    batch_loop<V, R, false>(blob, states, mats, parts, energies, grads, ctrl, timeout_ns);
}

// ------------------------------------------------------------------ host side
size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

bool pass_needs_big(const qs_pass& ps, const qs_op* ops) {
    for (int i = 0; i < ps.op_count; ++i) {
        const qs_op& op = ops[ps.op_begin + i];
        const bool diag = op.kind == QS_OP_DIAG || (op.kind == QS_OP_EXPECT && (op.flags & QS_OPF_DIAG));
        if (op.m >= 3 && !diag) return true;
        const bool dense = op.kind == QS_OP_MAT ||
                           ((op.kind == QS_OP_ANTI || op.kind == QS_OP_SWAP) && !(op.flags & QS_OPF_UNIT));
        if (dense && op.lctrl != 0) return true;
    }
    return false;
}

struct Stage {
    int32_t kind;   // BI_*
    int32_t args;   // FWD / BWD: BArgs index
    uint64_t size;  // FWD / BWD: tiles; HAM: amplitudes
    int fresh;
};

uint64_t fnv64(const std::string& t, uint64_t h = 1469598103934665603ull) {
    for (unsigned char c : t) h = (h ^ c) * 1099511628211ull;
    return h;
}

// Generated register-stage functions of planned batches, by the plan's
// jit_key: compile-cache keys of the functions (in dispatcher index order)
// and the dispatcher source.
struct BatchFns {
    std::vector<std::string> keys;
    std::string dispatcher;
};
std::mutex g_fns_mu;
std::unordered_map<uint64_t, std::shared_ptr<BatchFns>> g_fns;

std::string dispatcher_source(const std::vector<std::string>& names, bool c128) {
    std::string d = "typedef unsigned long long u64;\ntypedef unsigned int u32;\n";
    d += c128 ? "typedef double2 V;\n" : "typedef float2 V;\n";
    for (const auto& n : names)
        d += "extern \"C\" __device__ void " + n + "(V*, const void*, const V*, double*, u64, u64, u32);\n";
    d += "extern \"C\" __device__ int qs_batch_jit(int fn, void* vec, const void* params, const void* mats, "
         "double* partials, u64 t0, u64 t1, u32 zero_in) {\n  switch (fn) {\n";
    for (size_t i = 0; i < names.size(); ++i)
        d += "  case " + std::to_string(i) + ": " + names[i] +
             "((V*)vec, params, (const V*)mats, partials, t0, t1, zero_in); return 1;\n";
    d += "  default: return 0;\n  }\n}\n";
    return d;
}

}  // namespace
}  // namespace qs

using namespace qs;

extern "C" const unsigned long long qs_batch_dev_cubin_size;
extern "C" const unsigned char qs_batch_dev_cubin[];

extern "C" int qs_batch_plan(int dtype, const qs_batch_inst* inst, int ninst, const qs_pass* passes, int npasses,
                             const qs_op* ops, int64_t nops, int64_t mats_count, const void* mats_host,
                             int jit_min_qubits, const uint64_t* xmask,
                             const uint64_t* zmask, const double* coeff, int nterms_total, const double* weights,
                             int64_t nweights, int64_t tiles_per_item, int64_t amps_per_ham_item, void* blob,
                             size_t blob_bytes, qs_batch_sizes* sizes, int64_t* state_off) {
    QS_REQUIRE(valid_dtype(dtype), "bad dtype %d", dtype);
    QS_REQUIRE(inst != nullptr && ninst >= 1 && ninst <= (1 << 20), "instance count %d outside [1, 2^20]", ninst);
    QS_REQUIRE(passes != nullptr && ops != nullptr && sizes != nullptr, "null argument");
    QS_REQUIRE(nterms_total >= 1 && xmask != nullptr && zmask != nullptr && coeff != nullptr, "no observable terms");
    QS_REQUIRE(nweights >= 0 && (nweights == 0 || weights != nullptr), "null weights");
    QS_REQUIRE(tiles_per_item >= 1 && amps_per_ham_item >= 32, "item sizes must be >= 1 tile / 32 amplitudes");
    const int R = dtype == QS_C128 ? 4 : 5;  // register bits of the generic register kernel
    const int nb = dtype == QS_C128 ? 3 : 4;
    std::vector<BInst> bi(static_cast<size_t>(ninst));
    std::vector<std::vector<Stage>> stages(static_cast<size_t>(ninst));
    std::vector<std::vector<unsigned char>> arg_blobs;  // one compact record per register stage
    std::vector<BTerm> terms;
    std::vector<double> wts;
    int big = 0, maxnt = 5;
    std::vector<std::string> fn_names, fn_srcs;  // generated register-stage functions
    std::unordered_map<std::string, int> fn_index;
    size_t smem = 0;
    int64_t state_elems = 0, part_doubles = 0, grad_doubles = 0;
    static thread_local RegArgs ra;
    for (int i = 0; i < ninst; ++i) {
        const qs_batch_inst& q = inst[i];
        QS_REQUIRE(q.n >= 1 && q.n <= 34, "instance %d: qubit count %d outside [1, 34]", i, q.n);
        QS_REQUIRE(q.nfwd >= 1 && q.fwd_begin >= 0 && int64_t(q.fwd_begin) + q.nfwd <= npasses,
                   "instance %d: forward pass range outside the pass array (at least one pass)", i);
        QS_REQUIRE(q.nbwd >= 0 && q.bwd_begin >= 0 && int64_t(q.bwd_begin) + q.nbwd <= npasses,
                   "instance %d: backward pass range outside the pass array", i);
        QS_REQUIRE(q.nterms >= 1 && q.nterms <= 128 && q.term_begin >= 0 && q.term_begin + q.nterms <= nterms_total,
                   "instance %d: observable term range (1..128 terms) outside the term arrays", i);
        QS_REQUIRE(q.nslots >= 0 && q.nparams >= 0 && (q.nslots > 0 || q.nbwd == 0),
                   "instance %d: backward passes need EXPECT slots", i);
        QS_REQUIRE(q.w_begin >= 0 && q.w_begin + int64_t(q.nparams) * q.nslots <= nweights,
                   "instance %d: weights outside the weight array", i);
        BInst& b = bi[size_t(i)];
        memset(&b, 0, sizeof(b));
        b.n = q.n;
        b.nslots = q.nslots;
        b.nparams = q.nparams;
        b.nterms = q.nterms;
        b.term_begin = int32_t(terms.size());
        b.state_off = state_elems;
        state_elems += int64_t(2) << q.n;
        b.grad_off = grad_doubles;
        grad_doubles += q.nparams;
        b.w_off = int64_t(wts.size());
        for (int64_t k = 0; k < int64_t(q.nparams) * q.nslots; ++k) wts.push_back(weights[q.w_begin + k]);
        // observable terms, stably sorted by X mask, with i^popc(x & z) folded in
        std::vector<int> order(static_cast<size_t>(q.nterms));
        for (int t = 0; t < q.nterms; ++t) {
            const int g = q.term_begin + t;
            QS_REQUIRE((xmask[g] >> q.n) == 0 && (zmask[g] >> q.n) == 0, "instance %d: term %d acts on bits >= n", i, t);
            order[size_t(t)] = g;
        }
        std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return xmask[a] < xmask[c]; });
        for (int g : order) {
            BTerm tm;
            tm.x = xmask[g];
            tm.z = zmask[g];
            double re = coeff[2 * g], im = coeff[2 * g + 1];
            for (int k = 0; k < (__builtin_popcountll(xmask[g] & zmask[g]) & 3); ++k) {
                const double r2 = -im, i2 = re;
                re = r2;
                im = i2;
            }
            tm.cre = re;
            tm.cim = im;
            terms.push_back(tm);
        }
        // register stages
        int bwd_k = -1;
        for (int dir = 0; dir < 2; ++dir) {
            const bool bwd = dir == 1;
            const int nbits = bwd ? q.n + 1 : q.n;
            const int begin = bwd ? q.bwd_begin : q.fwd_begin, count = bwd ? q.nbwd : q.nfwd;
            for (int pi = 0; pi < count; ++pi) {
                const qs_pass& ps = passes[begin + pi];
                if (bwd) {
                    QS_REQUIRE(ps.pair == q.n + 1, "instance %d: backward pass %d must be a pair pass (pair bit n)", i, pi);
                    if (bwd_k < 0) bwd_k = ps.k;
                    QS_REQUIRE(ps.k == bwd_k, "instance %d: backward passes must share one tile width", i);
                } else {
                    QS_REQUIRE(ps.pair == 0, "instance %d: forward pass %d has a pair bit", i, pi);
                }
                const int64_t ntiles = int64_t(1) << (nbits - ps.k);
                int rc = validate_pass(ps, nbits, ops, nops, mats_count, bwd, 2 * int64_t(q.nslots) * ntiles);
                if (rc) return rc;
                const int nT = ps.k - R;
                if (!(nT >= 5 && nT <= 8 && ps.nlow >= 5)) {
                    set_error("instance %d: pass %d (tile 2^%d, nlow %d) is not a register tile of the batch kernel", i,
                              pi, ps.k, ps.nlow);
                    return QS_ENOTSUP;
                }
                if (bwd)
                    for (int o = 0; o < ps.op_count; ++o) {
                        const qs_op& op = ops[ps.op_begin + o];
                        const bool diag = op.kind == QS_OP_DIAG || (op.kind == QS_OP_EXPECT && (op.flags & QS_OPF_DIAG));
                        QS_REQUIRE(op.m <= 2 || diag, "instance %d: backward pass ops act densely on at most 2 bits", i);
                    }
                if (pass_needs_big(ps, ops)) {
                    set_error("instance %d: pass %d has dense ops on 3-4 bits or controlled dense ops, which the "
                              "batch kernel does not take", i, pi);
                    return QS_ENOTSUP;
                }
                QS_REQUIRE(ps.op_count > 0, "instance %d: pass %d has no ops", i, pi);
                std::vector<int> rem(static_cast<size_t>(ps.op_count));
                for (int o = 0; o < ps.op_count; ++o) rem[size_t(o)] = o;
                while (!rem.empty()) {  // a pass may need several register launches
                    if (build_reg(ps, ops, rem, nbits, R, nb, ra) <= 0) {
                        set_error("instance %d: an op of pass %d does not fit a register tile", i, pi);
                        return QS_EINVAL;
                    }
                    const size_t need = dtype == QS_C128 ? reg_smem_bytes<double2>(ra, R, bwd)
                                                         : reg_smem_bytes<float2>(ra, R, bwd);
                    smem = std::max(smem, need);
                    maxnt = std::max(maxnt, ra.nT);
                    // a generated function for the linked kernel (large problems)
                    int32_t jit_fn = -1;
                    std::vector<uint64_t> params;
                    if (mats_host != nullptr && q.n >= jit_min_qubits) {
                        static const char kSlot[] = "qs_pf_name_slot";
                        std::string src;
                        size_t jsmem = 0;
                        int jthreads = 0;
                        if (gen_batch_pass(&ra, R, dtype == QS_C128, mats_host, kSlot, &src, &params, &jsmem,
                                           &jthreads)) {
                            // the function's name: a hash of its text (equal passes share one function)
                            char nm[40];
                            snprintf(nm, sizeof(nm), "qs_pf_%016llx%c", (unsigned long long)fnv64(src),
                                     dtype == QS_C128 ? 'd' : 's');
                            for (size_t at = src.find(kSlot); at != std::string::npos; at = src.find(kSlot, at))
                                src.replace(at, sizeof(kSlot) - 1, nm);
                            auto f = fn_index.find(nm);
                            if (f == fn_index.end()) {
                                f = fn_index.emplace(nm, int(fn_names.size())).first;
                                fn_names.push_back(nm);
                                fn_srcs.push_back(std::move(src));
                            }
                            jit_fn = f->second;
                            smem = std::max(smem, jsmem);
                            maxnt = std::max(maxnt, 31 - __builtin_clz(unsigned(jthreads)));
                        } else {
                            params.clear();
                        }
                    }
                    // compact record: BArgs, then stages, ops, copies, EXPECT slots, parameter block
                    const size_t o_st = align16(sizeof(BArgs));
                    const size_t o_ops = align16(o_st + sizeof(KStage) * size_t(ra.nstages));
                    const size_t o_cp = align16(o_ops + sizeof(KOp) * size_t(ra.nops));
                    const size_t o_es = align16(o_cp + sizeof(KCopy) * size_t(ra.nops));
                    const size_t o_pb = align16(o_es + sizeof(int) * size_t(ra.nexp > 0 ? ra.nexp : 1));
                    const size_t tot = align16(o_pb + sizeof(uint64_t) * params.size());
                    std::vector<unsigned char> rec(tot, 0);
                    BArgs ba;
                    memset(&ba, 0, sizeof(ba));
                    ba.h = static_cast<const RegHead&>(ra);
                    ba.off_st = int64_t(o_st);  // relative here; made absolute when the blob is laid out
                    ba.off_ops = int64_t(o_ops);
                    ba.off_cp = int64_t(o_cp);
                    ba.off_es = int64_t(o_es);
                    ba.jit_fn = jit_fn;
                    ba.off_params = int64_t(o_pb);
                    if (!params.empty()) memcpy(rec.data() + o_pb, params.data(), sizeof(uint64_t) * params.size());
                    memcpy(rec.data(), &ba, sizeof(ba));
                    memcpy(rec.data() + o_st, ra.st, sizeof(KStage) * size_t(ra.nstages));
                    memcpy(rec.data() + o_ops, ra.ops, sizeof(KOp) * size_t(ra.nops));
                    memcpy(rec.data() + o_cp, ra.cp, sizeof(KCopy) * size_t(ra.nops));
                    if (ra.nexp > 0) memcpy(rec.data() + o_es, ra.eslot, sizeof(int) * size_t(ra.nexp));
                    Stage sg;
                    sg.kind = bwd ? BI_BWD : BI_FWD;
                    sg.args = int32_t(arg_blobs.size());
                    sg.size = uint64_t(ntiles);
                    sg.fresh = (!bwd && stages[size_t(i)].empty()) ? 1 : 0;
                    arg_blobs.push_back(std::move(rec));
                    stages[size_t(i)].push_back(sg);
                }
            }
            if (!bwd) {  // the HAM stage sits between the forward and the backward passes
                Stage sg;
                sg.kind = BI_HAM;
                sg.args = -1;
                sg.size = uint64_t(1) << q.n;
                sg.fresh = 0;
                stages[size_t(i)].push_back(sg);
            }
        }
        b.tiles_bwd = bwd_k < 0 ? 0 : int32_t(int64_t(1) << (q.n + 1 - bwd_k));
        Stage fin;
        fin.kind = BI_FIN;
        fin.args = -1;
        fin.size = 1;
        fin.fresh = 0;
        stages[size_t(i)].push_back(fin);
        smem = std::max(smem, sizeof(double) * size_t(q.nslots) + 16);
    }
    // items, round-robin over the instances by stage index, larger instances first
    std::vector<int> ord(static_cast<size_t>(ninst));
    for (int i = 0; i < ninst; ++i) ord[size_t(i)] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int c) {
        const double wa = std::ldexp(double(stages[size_t(a)].size()), inst[a].n);
        const double wc = std::ldexp(double(stages[size_t(c)].size()), inst[c].n);
        return wa > wc;
    });
    // Problems are interleaved in groups of `group` (default: all of them).
    // Smaller groups run fewer distinct stage functions at once, but cover the
    // tail of each stage with fewer other problems; on the 512-instance QAOA
    // batch (B200) all / 64 / 16 / 4 / 1 took 619 / 623 / 638 / 720 / 980 ms.
    // QS_BATCH_GROUP sets it (0: all).
    int group = ninst;
    if (const char* e = getenv("QS_BATCH_GROUP"))
        if (*e && atoi(e) > 0) group = atoi(e);
    std::vector<BItem> items;
    std::vector<int64_t> issued(size_t(ninst), 0);
    for (int g0 = 0; g0 < ninst; g0 += group) {
      const int g1 = std::min(ninst, g0 + group);
      size_t maxst = 0;
      for (int k = g0; k < g1; ++k) maxst = std::max(maxst, stages[size_t(ord[size_t(k)])].size());
      for (size_t r = 0; r < maxst; ++r)
        for (int k = g0; k < g1; ++k) {
            const int i = ord[size_t(k)];
            if (r >= stages[size_t(i)].size()) continue;
            const Stage& sg = stages[size_t(i)][r];
            const int64_t need = issued[size_t(i)];
            uint64_t step = 1, total = sg.size;
            if (sg.kind == BI_FWD || sg.kind == BI_BWD) step = uint64_t(tiles_per_item);
            else if (sg.kind == BI_HAM) step = uint64_t(amps_per_ham_item);
            int32_t idx = 0;
            for (uint64_t a = 0; a < total; a += step, ++idx) {
                BItem it;
                memset(&it, 0, sizeof(it));
                it.kind = sg.kind;
                it.inst = i;
                it.stage = sg.kind == BI_HAM ? idx : sg.args;
                it.fresh = sg.fresh;
                it.need = need;
                it.t0 = a;
                it.t1 = std::min(total, a + step);
                items.push_back(it);
                ++issued[size_t(i)];
            }
            if (sg.kind == BI_HAM) bi[size_t(i)].nham = idx;
        }
    }
    QS_REQUIRE(items.size() < size_t(1) << 31, "too many work items (%zu)", items.size());
    for (int i = 0; i < ninst; ++i) {
        BInst& b = bi[size_t(i)];
        b.part_off = part_doubles;
        part_doubles += 2 * int64_t(b.nslots) * b.tiles_bwd + 2 * int64_t(b.nham);
    }
    // blob layout
    const size_t o_items = align16(sizeof(BHead));
    const size_t o_inst = align16(o_items + sizeof(BItem) * items.size());
    const size_t o_args = align16(o_inst + sizeof(BInst) * size_t(ninst));
    size_t o_rec = align16(o_args + sizeof(BArgs) * arg_blobs.size());
    std::vector<size_t> rec_at(arg_blobs.size());
    for (size_t k = 0; k < arg_blobs.size(); ++k) {
        rec_at[k] = o_rec;
        o_rec = align16(o_rec + arg_blobs[k].size());
    }
    const size_t o_terms = o_rec;
    const size_t o_w = align16(o_terms + sizeof(BTerm) * terms.size());
    const size_t total = align16(o_w + sizeof(double) * (wts.empty() ? 1 : wts.size()));
    const int threads = 1 << maxnt;
    QS_REQUIRE(smem <= size_t(smem_optin()), "the batch needs %zu bytes of shared memory per CTA", smem);
    sizes->blob_bytes = int64_t(total);
    sizes->state_elems = state_elems;
    sizes->partial_doubles = part_doubles > 0 ? part_doubles : 1;
    sizes->grad_doubles = grad_doubles > 0 ? grad_doubles : 1;
    sizes->energy_doubles = 2 * int64_t(ninst);
    sizes->ctrl_bytes = int64_t(sizeof(unsigned long long)) * (kCtrlHead + ninst);
    sizes->smem_bytes = int64_t(smem);
    sizes->threads = threads;
    sizes->nitems = int32_t(items.size());
    sizes->nstages = int32_t(arg_blobs.size());
    sizes->big = big;
    sizes->dtype = dtype;
    sizes->jit_fns = int32_t(fn_names.size());
    {
        uint64_t key = fnv64(dtype == QS_C128 ? "c128" : "c64");
        for (const auto& nm : fn_names) key = fnv64(nm, key);
        sizes->jit_key = fn_names.empty() ? 0 : key;
    }
    if (state_off != nullptr)
        for (int i = 0; i < ninst; ++i) state_off[i] = bi[size_t(i)].state_off;
    if (blob == nullptr) return QS_OK;  // size query
    if (blob_bytes < total) {
        set_error("qs_batch_plan: the plan needs %zu bytes", total);
        return QS_EWORKSPACE;
    }
    unsigned char* out = static_cast<unsigned char*>(blob);
    memset(out, 0, total);
    BHead hd;
    memset(&hd, 0, sizeof(hd));
    hd.ninst = ninst;
    hd.nitems = int32_t(items.size());
    hd.nstages = int32_t(arg_blobs.size());
    hd.dtype = dtype;
    hd.threads = threads;
    hd.big = big;
    hd.off_items = int64_t(o_items);
    hd.off_inst = int64_t(o_inst);
    hd.off_args = int64_t(o_args);
    hd.off_terms = int64_t(o_terms);
    hd.off_w = int64_t(o_w);
    hd.smem = int64_t(smem);
    memcpy(out, &hd, sizeof(hd));
    if (!items.empty()) memcpy(out + o_items, items.data(), sizeof(BItem) * items.size());
    memcpy(out + o_inst, bi.data(), sizeof(BInst) * size_t(ninst));
    for (size_t k = 0; k < arg_blobs.size(); ++k) {
        BArgs ba;
        memcpy(&ba, arg_blobs[k].data(), sizeof(ba));
        ba.off_st += int64_t(rec_at[k]);
        ba.off_ops += int64_t(rec_at[k]);
        ba.off_cp += int64_t(rec_at[k]);
        ba.off_es += int64_t(rec_at[k]);
        ba.off_params += int64_t(rec_at[k]);
        memcpy(out + o_args + sizeof(BArgs) * k, &ba, sizeof(ba));
        memcpy(out + rec_at[k], arg_blobs[k].data(), arg_blobs[k].size());
    }
    if (!terms.empty()) memcpy(out + o_terms, terms.data(), sizeof(BTerm) * terms.size());
    if (!wts.empty()) memcpy(out + o_w, wts.data(), sizeof(double) * wts.size());
    if (!fn_names.empty()) {  // queue the functions' compilation (host threads) and record the batch
        auto b = std::make_shared<BatchFns>();
        for (size_t k = 0; k < fn_names.size(); ++k) {
            b->keys.push_back(jit::queue_device_fn(fn_srcs[k], fn_names[k].c_str()));
            if (b->keys.back().empty()) {
                set_error("qs_batch_plan: run-time compilation is unavailable: %s", jit::last_log());
                return QS_ENOTSUP;
            }
        }
        b->dispatcher = dispatcher_source(fn_names, dtype == QS_C128);
        std::lock_guard<std::mutex> lock(g_fns_mu);
        g_fns[sizes->jit_key] = b;
    }
    return QS_OK;
}

namespace {
// The linked kernel of a plan with generated functions, when it can run now
// (null: run the generic kernel).  Outside stream capture the first launch
// links and loads it (after the compilations in mode QS_JIT_SYNC; in mode
// QS_JIT_ASYNC only once they are done).
void* linked_kernel(const qs_batch_sizes& sz, cudaStream_t st, int* occ) {
    if (sz.jit_fns <= 0 || jit::mode() == QS_JIT_OFF) return nullptr;
    std::shared_ptr<BatchFns> b;
    {
        std::lock_guard<std::mutex> lock(g_fns_mu);
        auto it = g_fns.find(sz.jit_key);
        if (it == g_fns.end()) return nullptr;
        b = it->second;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) cs = cudaStreamCaptureStatusActive;
    const bool capturing = cs != cudaStreamCaptureStatusNone;
    return jit::link_module(sz.jit_key, qs_batch_dev_cubin, size_t(qs_batch_dev_cubin_size), b->dispatcher, b->keys,
                            sz.dtype == QS_C128 ? "qs_batch_linked_c128" : "qs_batch_linked_c64",
                            jit::mode() == QS_JIT_SYNC && !capturing, !capturing, sz.threads, size_t(sz.smem_bytes),
                            occ);
}

template <typename V, int R>
int launch_batch(const qs_batch_sizes& sz, const void* blob, void* states, const void* mats, double* parts,
                 double* energies, double* grads, void* ctrl, uint64_t timeout_ns, cudaStream_t st) {
    auto* fn = k_batch<V, R>;
    config_smem((const void*)fn);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, sz.threads, size_t(sz.smem_bytes));
    if (occ < 1) {
        set_error("qs_batch_launch: %d threads with %lld bytes of shared memory do not fit an SM", sz.threads,
                  (long long)sz.smem_bytes);
        return QS_ENOTSUP;
    }
    int locc = 0;
    void* lfn = linked_kernel(sz, st, &locc);
    if (lfn != nullptr) occ = locc;
    int64_t grid = int64_t(sm_count()) * occ;
    if (grid > sz.nitems) grid = sz.nitems;
    cudaError_t e = cudaMemsetAsync(ctrl, 0, size_t(sz.ctrl_bytes), st);
    if (e != cudaSuccess) {
        set_error("qs_batch_launch: cudaMemsetAsync: %s", cudaGetErrorString(e));
        return QS_ECUDA;
    }
    if (lfn != nullptr) {
        const unsigned char* b = static_cast<const unsigned char*>(blob);
        const void* m = mats;
        void* c = ctrl;
        void* params[] = {&b, &states, &m, &parts, &energies, &grads, &c, &timeout_ns};
        const int rc = jit::launch(lfn, unsigned(grid), unsigned(sz.threads), size_t(sz.smem_bytes), st, params);
        return rc ? rc : 1;
    }
    fn<<<unsigned(grid), unsigned(sz.threads), size_t(sz.smem_bytes), st>>>(
        static_cast<const unsigned char*>(blob), static_cast<V*>(states), static_cast<const V*>(mats), parts, energies,
        grads, static_cast<unsigned long long*>(ctrl), timeout_ns);
    QS_CHECK_LAUNCH("qs_batch_launch");
    return QS_OK;
}
}  // namespace

extern "C" int qs_batch_link_check(const qs_batch_sizes* sizes, int64_t* cubin_bytes) {
    QS_REQUIRE(sizes != nullptr && cubin_bytes != nullptr, "null argument");
    *cubin_bytes = 0;
    if (sizes->jit_fns <= 0) return QS_OK;
    std::shared_ptr<BatchFns> b;
    {
        std::lock_guard<std::mutex> lock(g_fns_mu);
        auto it = g_fns.find(sizes->jit_key);
        QS_REQUIRE(it != g_fns.end(), "qs_batch_link_check: the plan's functions are not registered");
        b = it->second;
    }
    const std::string cubin =
        jit::link_cubin(qs_batch_dev_cubin, size_t(qs_batch_dev_cubin_size), b->dispatcher, b->keys, true);
    if (cubin.empty()) {
        set_error("qs_batch_link_check: %s", jit::last_log());
        return QS_ENOTSUP;
    }
    *cubin_bytes = int64_t(cubin.size());
    return QS_OK;
}

extern "C" int qs_batch_launch(const qs_batch_sizes* sizes, const void* blob_dev, void* states, const void* mats,
                               double* partials, double* energies, double* grads, void* ctrl, size_t ctrl_bytes,
                               double timeout_s, void* stream) {
    QS_REQUIRE(sizes != nullptr && blob_dev != nullptr && states != nullptr && mats != nullptr && partials != nullptr &&
                   energies != nullptr && grads != nullptr && ctrl != nullptr,
               "null argument");
    QS_REQUIRE(valid_dtype(sizes->dtype), "bad dtype %d in the plan sizes", sizes->dtype);
    QS_REQUIRE(ctrl_bytes >= size_t(sizes->ctrl_bytes), "control buffer needs %lld bytes", (long long)sizes->ctrl_bytes);
    QS_REQUIRE(sizes->threads >= 32 && sizes->threads <= 256 && sizes->nitems >= 1, "bad plan sizes");
    QS_REQUIRE((reinterpret_cast<uintptr_t>(blob_dev) & 15) == 0, "the plan must be 16-byte aligned on the device");
    QS_REQUIRE(timeout_s > 0 && timeout_s <= 600, "timeout %g s outside (0, 600]", timeout_s);
    const uint64_t tns = uint64_t(timeout_s * 1e9);
    cudaStream_t st = as_stream(stream);
    QS_REQUIRE(sizes->big == 0, "the batch kernel takes no dense ops on 3-4 bits or controlled dense ops");
    if (sizes->dtype == QS_C128)
        return launch_batch<double2, 4>(*sizes, blob_dev, states, mats, partials, energies, grads, ctrl, tns, st);
    return launch_batch<float2, 5>(*sizes, blob_dev, states, mats, partials, energies, grads, ctrl, tns, st);
}
