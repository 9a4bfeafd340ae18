// library.cu -- host orchestration and the explicit C ABI of libpatgpu.so:
// basis snapshot, shell pairs, Schwarz bounds, class-sorted screened quartet
// lists, and the Fock builds that launch the class kernels of eri.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdarg>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/patgpu.h"
#include "eri.cuh"
#include "eri_grad.cuh"
#include "onebody.cuh"
#include "rys_table.h"

namespace pg {

// ------------------------------------------------------------------ errors
static thread_local int t_err = 0;
static thread_local char t_msg[512] = "";

int fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_msg, sizeof(t_msg), fmt, ap);
    va_end(ap);
    t_err = code;
    return code;
}

#define PG_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail(PATGPU_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------ device memory
struct DBuf {
    void *p = nullptr;
    size_t bytes = 0;
    ~DBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t ensure(size_t b)
    {
        if (b <= bytes && p) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, b ? b : 16);
        if (e == cudaSuccess) bytes = b;
        return e;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

template <class T>
static cudaError_t upload(DBuf &b, const std::vector<T> &v, cudaStream_t s)
{
    cudaError_t e = b.ensure(sizeof(T) * v.size());
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s);
}

// ------------------------------------------------------------------ tables
// Rys coefficients and constant tables, uploaded once per device (a process
// may drive several GPUs, one handle per device)
constexpr int kMaxDevices = 64;
static std::mutex g_tab_lock;
static DBuf *g_rys_coef[kMaxDevices] = {};
static int g_tab_state[kMaxDevices] = {};   // 0 not yet, 1 uploaded, -1 failed

static RysConst host_rys_const()
{
    RysConst rc{};
    for (int n = 0; n <= RYS_NMAX; ++n) {
        rc.tmax[n] = rys_tmax[n];
        rc.off[n] = rys_off[n];
        for (int i = 0; i < RYS_NMAX; ++i) {
            rc.lag_x[n][i] = rys_lag_x[n][i];
            rc.lag_w[n][i] = rys_lag_w[n][i];
        }
    }
    return rc;
}

static int init_tables()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(PATGPU_ENODEV, "no usable current CUDA device");
    std::lock_guard<std::mutex> g(g_tab_lock);
    if (g_tab_state[dev] == 0) {
        auto *b = new DBuf();
        // the device keeps the coefficient-major copy (rys_eval, interleaved)
        std::vector<double> il(rys_ncoef);
        rys_interleave(rys_coef_host, il.data(), rys_off, rys_tmax, RYS_NMAX, RYS_DEG);
        const bool ok =
            b->ensure(sizeof(double) * rys_ncoef) == cudaSuccess &&
            cudaMemcpy(b->p, il.data(), sizeof(double) * rys_ncoef, cudaMemcpyHostToDevice) == cudaSuccess &&
            upload_rys_constants(host_rys_const()) == cudaSuccess && upload_onebody_constants() == cudaSuccess;
        g_rys_coef[dev] = b;
        g_tab_state[dev] = ok ? 1 : -1;
    }
    if (g_tab_state[dev] < 0) return fail(PATGPU_ECUDA, "uploading the Rys tables to device %d failed", dev);
    return 0;
}

// ------------------------------------------------------------------ handle
struct ClassWork {
    int la, lb, lc, ld;
    long long offset, count;     // count: quartets this rank owns after screening
    int variant = 0;             // kernel variant chosen for this class (see tune_variants)
    int variant32 = 3;           // kernel of the mixed-precision window: FP32 (3, 4) or `variant` (see tune_fp32)
    int u0 = 0, nu = 0, v0 = 0, nv = 0, same = 0;   // bra and ket pair ranges
    long long total = 0;         // unscreened quartets of the class (all ranks)
    long long items = 0;         // work items of this rank: ceil((total - rank) / nranks)
    int idx = 0;                 // position in the handle's work list
    // compacted lists: this class's survivors at [loff, loff + count) of the
    // handle's list, the FP64 window (bound >= tau_mix, or all without mixed
    // precision) first, nhi entries, then the FP32 window
    long long loff = 0, nhi = 0;
};

static int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }

}  // namespace pg

struct patgpu_basis {
    // snapshot
    int nsh = 0, ncen = 0, n = 0, skipcen = 0;
    int dev = 0;                     // the device the handle's buffers live on
    std::vector<int> l, cen, off, nst, poff;
    std::vector<double> al, co, q, xyz;
    double tau = 0.0;
    double tau_mix = 0.0;            // > 0: quartets with bounds in [tau, tau_mix) run in FP32
    // 1: J/K accumulate as exact fixed-point integers (acc_add), so G is
    // bitwise reproducible; the accumulators then hold 16 bytes an element
    int det = 1;
    long long nquart_fp32 = 0;
    int start_shell = 0, rank = 0, nranks = 1;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    // pairs (class-sorted)
    int npair = 0;
    std::vector<int> psa, psb, pfa, pfb, pcls, pstart, pnum;
    std::vector<double> pax, pay, paz, pabx, paby, pabz, Q;
    std::vector<double> pp_p, pp_px, pp_py, pp_pz, pp_K, pp_cut;
    std::vector<int> pca, pcb;        // centres of the two shells (gradient)
    std::vector<double> pp_ea;        // exponent of the first shell's primitive (gradient)
    std::vector<int> class_begin;   // pairs of class c: [class_begin[c], class_begin[c+1])
    pg::DBuf d_psa, d_psb, d_pfa, d_pfb, d_pax, d_pay, d_paz, d_pabx, d_paby, d_pabz, d_pstart, d_pnum;
    pg::DBuf d_pp_p, d_pp_px, d_pp_py, d_pp_pz, d_pp_K, d_pp_cut, d_Q;
    pg::DBuf d_pca, d_pcb, d_pp_ea;
    pg::DBuf d_ppk;                  // packed pair records (one-primitive handles)
    // quartets
    std::vector<pg::ClassWork> work;
    long long nquart = 0, nquart_unscreened = 0;
    pg::DBuf d_list;                 // compacted class quartet indices (uint64), when lists are on
    bool lists = false;
    bool single_prim = false;        // every shell pair has exactly one primitive pair
    // density-weighted screening of host-buffer builds (tau_dens > 0): the
    // lists are filtered by Q_ab Q_cd max|D| against the build's density
    double tau_dens = 0.0;
    // > 0 with tau_dens: a kept quartet whose density-weighted bound is below
    // this runs in FP32 (the contribution, not just the integral, is small)
    double tau_dens32 = 0.0;
    pg::DBuf d_soff, d_snst, d_dsh, d_flist, d_fcnt;
    std::vector<unsigned long long> fcnt;   // per class: filtered FP64, FP32 sublist counts
    bool filtered = false;                  // the current build runs over d_flist
    // the filter reads its thresholds {tau_dens, tau_dens32} from device
    // memory (d_scr, or a batch's copy), so that a captured graph follows
    // threshold changes without being captured again
    pg::DBuf d_scr;
    // the launches of the density-weighted FP32 sublists are enqueued even
    // while tau_dens32 is 0 (they then run no quartet): a batch sets this
    // once its builds have used tau_dens32 > 0, so its graph stays valid
    bool dens32_armed = false;
    long long last_computed = 0;            // quartets computed by the last host-buffer build
    // work buffers
    pg::DBuf d_D0, d_D1, d_A0, d_A1, d_Pk0, d_Pk1, d_Gk0, d_Gk1, d_err;
    std::vector<double> h_stage;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ns = 0.0;
    int last_launches = 0;

    pg::EriArgs base_args() const
    {
        pg::EriArgs a{};
        a.pr.sa = d_psa.as<int>();
        a.pr.sb = d_psb.as<int>();
        a.pr.fa = d_pfa.as<int>();
        a.pr.fb = d_pfb.as<int>();
        a.pr.ax = d_pax.as<double>();
        a.pr.ay = d_pay.as<double>();
        a.pr.az = d_paz.as<double>();
        a.pr.abx = d_pabx.as<double>();
        a.pr.aby = d_paby.as<double>();
        a.pr.abz = d_pabz.as<double>();
        a.pr.pstart = d_pstart.as<int>();
        a.pr.pnum = d_pnum.as<int>();
        a.pp.p = d_pp_p.as<double>();
        a.pp.px = d_pp_px.as<double>();
        a.pp.py = d_pp_py.as<double>();
        a.pp.pz = d_pp_pz.as<double>();
        a.pp.K = d_pp_K.as<double>();
        a.pp.cut = d_pp_cut.as<double>();
        a.n = n;
        a.rys_coef = pg::g_rys_coef[dev]->as<double>();
        a.prim_cut = 1e-15;
        a.single_prim = single_prim ? 1 : 0;
        a.err = d_err.as<int>();
        a.det = det;
        a.ppk = single_prim ? d_ppk.as<double>() : nullptr;
        return a;
    }
};

namespace pg {

static int build_pairs(patgpu_basis *h)
{
    struct Tmp {
        int a, b, cls;
    };
    std::vector<Tmp> t;
    for (int i = 0; i < h->nsh; ++i) {
        if (!h->nst[i]) continue;
        for (int j = 0; j <= i; ++j) {
            if (!h->nst[j]) continue;
            int a = i, b = j;
            if (h->l[i] < h->l[j]) std::swap(a, b);   // larger l first (twoints.c:249-266)
            t.push_back({a, b, pair_class(h->l[a], h->l[b])});
        }
    }
    std::stable_sort(t.begin(), t.end(), [](const Tmp &x, const Tmp &y) { return x.cls < y.cls; });
    h->npair = (int)t.size();
    h->psa.clear(); h->psb.clear(); h->pfa.clear(); h->pfb.clear(); h->pcls.clear();
    h->pstart.clear(); h->pnum.clear(); h->pax.clear(); h->pay.clear(); h->paz.clear();
    h->pabx.clear(); h->paby.clear(); h->pabz.clear();
    h->pp_p.clear(); h->pp_px.clear(); h->pp_py.clear(); h->pp_pz.clear(); h->pp_K.clear(); h->pp_cut.clear();
    h->pca.clear(); h->pcb.clear(); h->pp_ea.clear();
    h->class_begin.assign(11, 0);
    for (auto &x : t) h->class_begin[x.cls + 1]++;
    for (int c = 0; c < 10; ++c) h->class_begin[c + 1] += h->class_begin[c];
    for (auto &x : t) {
        const double *A = &h->xyz[3 * h->cen[x.a]], *B = &h->xyz[3 * h->cen[x.b]];
        double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
        double ab2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
        h->psa.push_back(x.a);
        h->psb.push_back(x.b);
        h->pfa.push_back(h->off[x.a]);
        h->pfb.push_back(h->off[x.b]);
        h->pcls.push_back(x.cls);
        h->pca.push_back(h->cen[x.a]);
        h->pcb.push_back(h->cen[x.b]);
        h->pax.push_back(A[0]); h->pay.push_back(A[1]); h->paz.push_back(A[2]);
        h->pabx.push_back(AB[0]); h->paby.push_back(AB[1]); h->pabz.push_back(AB[2]);
        h->pstart.push_back((int)h->pp_p.size());
        int np = 0;
        for (int i = h->poff[x.a]; i < h->poff[x.a + 1]; ++i)
            for (int j = h->poff[x.b]; j < h->poff[x.b + 1]; ++j) {
                double ea = h->al[i], eb = h->al[j], p = ea + eb;
                double s = std::exp(-ea * eb * ab2 / p);
                h->pp_p.push_back(p);
                h->pp_px.push_back((ea * A[0] + eb * B[0]) / p);
                h->pp_py.push_back((ea * A[1] + eb * B[1]) / p);
                h->pp_pz.push_back((ea * A[2] + eb * B[2]) / p);
                h->pp_cut.push_back(s / p);
                h->pp_K.push_back(h->co[i] * h->co[j] * s / p);
                h->pp_ea.push_back(ea);
                ++np;
            }
        h->pnum.push_back(np);
    }
    h->single_prim = true;
    for (int np : h->pnum) h->single_prim = h->single_prim && np == 1;
    cudaStream_t s = h->stream;
    cudaError_t e = cudaSuccess;
#define UP(buf, vec) if (e == cudaSuccess) e = upload(h->buf, h->vec, s)
    UP(d_psa, psa); UP(d_psb, psb); UP(d_pfa, pfa); UP(d_pfb, pfb);
    UP(d_pax, pax); UP(d_pay, pay); UP(d_paz, paz); UP(d_pabx, pabx); UP(d_paby, paby); UP(d_pabz, pabz);
    UP(d_pstart, pstart); UP(d_pnum, pnum);
    UP(d_pp_p, pp_p); UP(d_pp_px, pp_px); UP(d_pp_py, pp_py); UP(d_pp_pz, pp_pz); UP(d_pp_K, pp_K);
    UP(d_pp_cut, pp_cut);
    UP(d_pca, pca); UP(d_pcb, pcb); UP(d_pp_ea, pp_ea);
    if (h->single_prim) {
        // one 128-byte record per pair (EriArgs::ppk)
        std::vector<double> pk(16 * (size_t)h->npair, 0.0);
        for (int u = 0; u < h->npair; ++u) {
            double *r = &pk[16 * (size_t)u];
            const int ip = h->pstart[u];
            r[0] = h->pp_p[ip]; r[1] = h->pp_px[ip]; r[2] = h->pp_py[ip]; r[3] = h->pp_pz[ip];
            r[4] = h->pp_K[ip]; r[5] = h->pp_cut[ip];
            r[6] = h->pax[u]; r[7] = h->pay[u]; r[8] = h->paz[u];
            r[9] = h->pabx[u]; r[10] = h->paby[u]; r[11] = h->pabz[u];
            const unsigned long long f = (unsigned long long)(unsigned)h->pfa[u] |
                                         ((unsigned long long)(unsigned)h->pfb[u] << 32);
            const unsigned long long sh = (unsigned long long)(unsigned)h->psa[u] |
                                          ((unsigned long long)(unsigned)h->psb[u] << 32);
            memcpy(&r[12], &f, 8);
            memcpy(&r[13], &sh, 8);
        }
        if (e == cudaSuccess) e = upload(h->d_ppk, pk, s);
    }
#undef UP
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(PATGPU_ECUDA, "pair upload: %s", cudaGetErrorString(e));
    return 0;
}

static void class_ls(int cls, int &la, int &lb)
{
    la = 0;
    while ((la + 1) * (la + 2) / 2 <= cls) ++la;
    lb = cls - la * (la + 1) / 2;
}

// Run export-mode kernels over explicit (u, v) pair quartets; out receives
// the blocks in kernel orientation at the offsets returned in offs.
static int export_pairs(patgpu_basis *h, const std::vector<int2> &quart, std::vector<double> &out,
                        std::vector<long long> &offs, double prim_cut = 1e-15)
{
    // group by class pair, keep the caller's order inside each group
    const size_t nq = quart.size();
    offs.assign(nq, 0);
    long long total = 0;
    std::vector<size_t> order(nq);
    for (size_t i = 0; i < nq; ++i) order[i] = i;
    auto key = [&](size_t i) { return h->pcls[quart[i].x] * 16 + h->pcls[quart[i].y]; };
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return key(x) < key(y); });
    std::vector<int2> sorted(nq);
    std::vector<long long> soff(nq);
    for (size_t k = 0; k < nq; ++k) {
        size_t i = order[k];
        sorted[k] = quart[i];
        int la, lb, lc, ld;
        class_ls(h->pcls[quart[i].x], la, lb);
        class_ls(h->pcls[quart[i].y], lc, ld);
        soff[k] = total;
        offs[i] = total;
        total += (long long)ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
    }
    DBuf dq, dout, doff;
    cudaStream_t s = h->stream;
    PG_CUDA(upload(dq, sorted, s));
    PG_CUDA(upload(doff, soff, s));
    PG_CUDA(dout.ensure(sizeof(double) * (size_t)std::max<long long>(total, 1)));
    size_t k = 0;
    while (k < nq) {
        size_t e = k;
        while (e < nq && key(order[e]) == key(order[k])) ++e;
        int la, lb, lc, ld;
        class_ls(h->pcls[sorted[k].x], la, lb);
        class_ls(h->pcls[sorted[k].y], lc, ld);
        EriArgs a = h->base_args();
        a.mode = MODE_EXPORT;
        a.prim_cut = prim_cut;
        a.quart = dq.as<int2>() + k;
        a.nquart = (long long)(e - k);
        a.out = dout.as<double>();
        a.out_off = doff.as<long long>() + k;
        PG_CUDA(launch_eri_class(la, lb, lc, ld, a, s, h->num_sms));
        k = e;
    }
    out.resize((size_t)total);
    if (total) PG_CUDA(cudaMemcpyAsync(out.data(), dout.p, sizeof(double) * total, cudaMemcpyDeviceToHost, s));
    PG_CUDA(cudaStreamSynchronize(s));
    return 0;
}

static int build_schwarz(patgpu_basis *h)
{
    std::vector<int2> diag(h->npair);
    for (int u = 0; u < h->npair; ++u) diag[u] = make_int2(u, u);
    std::vector<double> out;
    std::vector<long long> offs;
    // no primitive cut here: a pair whose own diagonal falls below the cut
    // can still meet a diffuse pair above it, so its bound must be exact
    int rc = export_pairs(h, diag, out, offs, 0.0);
    if (rc) return rc;
    h->Q.assign(h->npair, 0.0);
    for (int u = 0; u < h->npair; ++u) {
        int la, lb;
        class_ls(h->pcls[u], la, lb);
        const int na = ncart(la), nb = ncart(lb);
        double m = 0.0;
        for (int i = 0; i < na; ++i)
            for (int j = 0; j < nb; ++j) {
                double v = out[offs[u] + (((size_t)i * nb + j) * na + i) * nb + j];
                m = std::max(m, std::fabs(v));
            }
        h->Q[u] = std::sqrt(m);
    }
    return 0;
}

// Arguments of the implicit (list-free) launch of class w: every work item
// maps to one bra x ket pair combination, screened on the device.
static EriArgs class_args(const patgpu_basis *h, const ClassWork &w, int mode, double tau_lo, double tau_hi)
{
    EriArgs a = h->base_args();
    a.mode = mode;
    a.implicit = 1;
    a.u0 = w.u0;
    a.nu = w.nu;
    a.v0 = w.v0;
    a.nv = w.nv;
    a.same = w.same;
    a.rank = h->rank;
    a.nranks = h->nranks;
    a.start_shell = h->start_shell;
    a.Q = h->d_Q.as<double>();
    a.tau_lo = tau_lo;
    a.tau_hi = tau_hi;
    a.nquart = w.items;
    return a;
}

// Launch the class kernel(s) of w with the densities, accumulators and mode
// carried by proto.
// With mixed precision on, the class runs twice over its pair space: the
// tuned FP64 kernel on the quartets whose bound is at least tau_mix, the FP32
// kernel on those between the screening threshold and tau_mix.
// Arguments over the compacted list of class w: window 0 = the FP64 part
// (everything without mixed precision), 1 = the FP32 part, 2 = all survivors.
static EriArgs list_args(const patgpu_basis *h, const ClassWork &w, int mode, int window)
{
    EriArgs a = class_args(h, w, mode, -1.0, INFINITY);
    if (h->filtered && window != 2) {
        // density-screened sublists of this build (density_filter): the FP64
        // part from the start of the class's region, the FP32 part at its end;
        // their lengths are read on the device
        a.klist = h->d_flist.as<unsigned long long>() + w.loff;
        a.nquart = w.count;
        a.nq_dev = h->d_fcnt.as<unsigned long long>() + 2 * w.idx + window;
        a.from_end = window == 1;
        return a;
    }
    const unsigned long long *l = h->d_list.as<unsigned long long>() + w.loff;
    a.klist = window == 1 ? l + w.nhi : l;
    a.nquart = window == 0 ? w.nhi : (window == 1 ? w.count - w.nhi : w.count);
    return a;
}

static cudaError_t launch_work(const patgpu_basis *h, const ClassWork &w, const EriArgs &proto, cudaStream_t s)
{
    const double lo = h->tau > 0.0 ? h->tau : -1.0;
    const bool mixed =
        (h->tau_mix > lo && h->tau_mix > 0.0) || (h->filtered && (h->tau_dens32 > 0.0 || h->dens32_armed));
    if (h->lists) {
        // a class whose FP32 window is kept on its FP64 kernel (tune_fp32)
        // runs both windows, adjacent in its unfiltered list, as one launch
        const bool fold = mixed && w.variant32 == w.variant && !h->filtered;
        EriArgs a = list_args(h, w, proto.mode, fold ? 2 : 0);
        a.D0 = proto.D0;
        a.D1 = proto.D1;
        a.A0 = proto.A0;
        a.A1 = proto.A1;
        if (a.nquart > 0) {
            cudaError_t e = launch_eri_class(w.la, w.lb, w.lc, w.ld, a, s, h->num_sms, w.variant);
            if (e != cudaSuccess) return e;
        }
        if (!mixed || fold) return cudaSuccess;
        a = list_args(h, w, proto.mode, 1);
        a.D0 = proto.D0;
        a.D1 = proto.D1;
        a.A0 = proto.A0;
        a.A1 = proto.A1;
        return a.nquart > 0 ? launch_eri_class(w.la, w.lb, w.lc, w.ld, a, s, h->num_sms, w.variant32)
                            : cudaSuccess;
    }
    // without lists every class runs FP64 over its whole window: a second
    // (FP32) pass over the implicit space would step every team through
    // all of the class's items again and cost more than it saves
    EriArgs a = class_args(h, w, proto.mode, lo, INFINITY);
    a.D0 = proto.D0;
    a.D1 = proto.D1;
    a.A0 = proto.A0;
    a.A1 = proto.A1;
    return launch_eri_class(w.la, w.lb, w.lc, w.ld, a, s, h->num_sms, w.variant);
}

__global__ void count_kernel(const EriArgs a, unsigned long long *cnt)
{
    unsigned long long c = 0;
    for (long long qi = (long long)blockIdx.x * blockDim.x + threadIdx.x; qi < a.nquart;
         qi += (long long)gridDim.x * blockDim.x) {
        int u, v;
        if (eri_quartet_at(a, qi, u, v)) ++c;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(cnt, c);
}

// Which quartets may run in FP32.  The Schwarz bound Q_ab Q_cd limits an
// integral, not the terms the Rys scheme sums to get it: for diffuse
// distributions far apart the roots' terms are many orders of magnitude
// larger than their sum (the sum is a high multipole; each term carries
// powers of the root-scaled P-Q distance), and FP32 rounding errors scale
// with the terms.  term_bound is an upper estimate of those terms for bra
// pair u and ket pair v of a class with la+lb = lab and lc+ld = lcd: per
// primitive pair, the prefactor 2 pi^(5/2) |K_ab K_cd| / sqrt(p+q) times
// (2|A-B| + q/(p+q)|P-Q| + sqrt((lab+1)/2p))^lab (every recursion and
// transfer entry of the bra side stays below this power; likewise the ket
// side), summed over primitive pairs.  The FP32 window is term_bound <
// tau_fp32, which keeps FP32 rounding near eps_32 * tau_fp32 per integral.
// Contracted pairs with more than 64 primitive-pair combinations stay FP64.
constexpr double kTermSR = 34.98683665524972497;   // 2 pi^(5/2)

__device__ double ipow_small(double x, int l)
{
    double r = 1.0;
    for (int i = 0; i < l; ++i) r *= x;
    return r;
}

__device__ double term_bound(const EriArgs &a, int u, int v, int lab, int lcd)
{
    const int pu = a.pr.pstart[u], nu = a.pr.pnum[u], pv = a.pr.pstart[v], nv = a.pr.pnum[v];
    if (nu * nv > 64) return INFINITY;
    const double abl = sqrt(a.pr.abx[u] * a.pr.abx[u] + a.pr.aby[u] * a.pr.aby[u] + a.pr.abz[u] * a.pr.abz[u]);
    const double cdl = sqrt(a.pr.abx[v] * a.pr.abx[v] + a.pr.aby[v] * a.pr.aby[v] + a.pr.abz[v] * a.pr.abz[v]);
    double e = 0.0;
    for (int ib = pu; ib < pu + nu; ++ib)
        for (int ik = pv; ik < pv + nv; ++ik) {
            const double p = a.pp.p[ib], q = a.pp.p[ik], ppq = p + q;
            const double dx = a.pp.px[ib] - a.pp.px[ik], dy = a.pp.py[ib] - a.pp.py[ik],
                         dz = a.pp.pz[ib] - a.pp.pz[ik];
            const double R = sqrt(dx * dx + dy * dy + dz * dz);
            const double sb = 2.0 * abl + q / ppq * R + sqrt((lab + 1) / (2.0 * p));
            const double sk = 2.0 * cdl + p / ppq * R + sqrt((lcd + 1) / (2.0 * q));
            e += kTermSR * fabs(a.pp.K[ib] * a.pp.K[ik]) * rsqrt(ppq) * ipow_small(sb, lab) * ipow_small(sk, lcd);
        }
    return e == e ? e : INFINITY;
}

// Stream compaction of one window of a class's implicit quartet space: the
// (bra pair, ket pair) of every surviving item, packed as u | v << 32 and
// appended at out[*cursor++] with
// warp-aggregated atomics (order within a warp kept).  With lab >= 0 an
// item is kept only when its term_bound lies in [elo, ehi) as well (the
// FP64 or the FP32 window of mixed precision).
__global__ void compact_kernel(const EriArgs a, unsigned long long *out, unsigned long long *cursor, int lab = -1,
                               int lcd = 0, double elo = 0.0, double ehi = 0.0)
{
    for (long long qi0 = (long long)blockIdx.x * blockDim.x; qi0 < a.nquart;
         qi0 += (long long)gridDim.x * blockDim.x) {
        const long long qi = qi0 + threadIdx.x;
        int u, v;
        bool keep = qi < a.nquart && eri_quartet_at(a, qi, u, v);
        if (keep && lab >= 0) {
            const double e = term_bound(a, u, v, lab, lcd);
            keep = e >= elo && e < ehi;
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (!m) continue;
        const int lane = threadIdx.x & 31, lead = __ffs(m) - 1;
        unsigned long long base = 0;
        if (lane == lead) base = atomicAdd(cursor, (unsigned long long)__popc(m));
        base = __shfl_sync(0xffffffffu, base, lead);
        if (keep)
            out[base + __popc(m & ((1u << lane) - 1u))] =
                (unsigned long long)(unsigned)u | ((unsigned long long)(unsigned)v << 32);
    }
}

// Compacted quartet lists (8 bytes per surviving quartet: bra pair | ket
// pair << 32), when they fit in
// half of the free device memory above a reserve of a tenth of the device
// and PATGPU_LISTS is not 0: the class
// kernels then visit only surviving quartets instead of stepping their
// teams through screened-out items.  With mixed precision on, each class's
// list is split into its FP64 and FP32 windows.
static int build_lists(patgpu_basis *h)
{
    h->lists = false;
    const char *env = getenv("PATGPU_LISTS");
    if (env && !strcmp(env, "0")) return 0;
    long long total = 0;
    for (auto &w : h->work) {
        w.loff = total;
        total += w.count;
    }
    size_t fr = 0, tot = 0;
    PG_CUDA(cudaMemGetInfo(&fr, &tot));
    // keep a tenth of the device (at least 4 GiB) out of reach of the lists,
    // so that many handles (a batch) cannot starve each other's set-up
    const size_t reserve = std::max<size_t>(tot / 10, (size_t)4 << 30);
    const size_t room = fr > reserve ? (fr - reserve) / 2 : 0;
    const size_t bytes = sizeof(unsigned long long) * (size_t)std::max<long long>(total, 1);
    if (bytes > h->d_list.bytes && bytes > room) {
        h->d_list.release();
        return 0;
    }
    PG_CUDA(h->d_list.ensure(bytes));
    const double lo = h->tau > 0.0 ? h->tau : -1.0;
    const bool mixed = h->tau_mix > lo && h->tau_mix > 0.0;
    DBuf dcur;
    const size_t nc = 2 * h->work.size();
    PG_CUDA(dcur.ensure(sizeof(unsigned long long) * std::max<size_t>(nc, 1)));
    PG_CUDA(cudaMemsetAsync(dcur.p, 0, sizeof(unsigned long long) * std::max<size_t>(nc, 1), h->stream));
    unsigned long long *out = h->d_list.as<unsigned long long>();
    for (size_t k = 0; k < h->work.size(); ++k) {
        const ClassWork &w = h->work[k];
        // FP64 window first (term_bound >= tau_mix), then the FP32 window
        // behind it; both screened by the Schwarz bound at tau
        EriArgs a = class_args(h, w, MODE_RHF, lo, INFINITY);
        const int g = (int)std::min<long long>((a.nquart + 255) / 256, (long long)h->num_sms * 16);
        if (mixed)
            compact_kernel<<<std::max(g, 1), 256, 0, h->stream>>>(a, out + w.loff, dcur.as<unsigned long long>() + 2 * k,
                                                                  w.la + w.lb, w.lc + w.ld, h->tau_mix, INFINITY);
        else
            compact_kernel<<<std::max(g, 1), 256, 0, h->stream>>>(a, out + w.loff, dcur.as<unsigned long long>() + 2 * k);
    }
    PG_CUDA(cudaGetLastError());
    std::vector<unsigned long long> cur(std::max<size_t>(nc, 1), 0);
    PG_CUDA(cudaMemcpyAsync(cur.data(), dcur.p, sizeof(unsigned long long) * cur.size(), cudaMemcpyDeviceToHost,
                            h->stream));
    PG_CUDA(cudaStreamSynchronize(h->stream));
    for (size_t k = 0; k < h->work.size(); ++k) h->work[k].nhi = (long long)cur[2 * k];
    if (mixed) {
        for (size_t k = 0; k < h->work.size(); ++k) {
            const ClassWork &w = h->work[k];
            EriArgs a = class_args(h, w, MODE_RHF, lo, INFINITY);
            const int g = (int)std::min<long long>((a.nquart + 255) / 256, (long long)h->num_sms * 16);
            compact_kernel<<<std::max(g, 1), 256, 0, h->stream>>>(a, out + w.loff + w.nhi,
                                                                  dcur.as<unsigned long long>() + 2 * k + 1,
                                                                  w.la + w.lb, w.lc + w.ld, -1.0, h->tau_mix);
        }
        PG_CUDA(cudaGetLastError());
        PG_CUDA(cudaMemcpyAsync(cur.data(), dcur.p, sizeof(unsigned long long) * cur.size(), cudaMemcpyDeviceToHost,
                                h->stream));
        PG_CUDA(cudaStreamSynchronize(h->stream));
    }
    for (size_t k = 0; k < h->work.size(); ++k) {
        const ClassWork &w = h->work[k];
        const long long got = (long long)cur[2 * k] + (mixed ? (long long)cur[2 * k + 1] : 0);
        if (got != w.count)
            return fail(PATGPU_ESTATE, "quartet list of class (%d%d|%d%d): %lld entries, %lld counted", w.la, w.lb,
                        w.lc, w.ld, got, w.count);
    }
    h->lists = true;
    return 0;
}

// Per class pair (bra class >= ket class): the pair ranges and the number of
// quartets that survive screening on this rank (counted on the device, so no
// quartet list is ever built; lists of 1e10 quartets would not fit).
static int build_quartets(patgpu_basis *h)
{
    h->work.clear();
    long long unscreened = 0, owned = 0;
    PG_CUDA(upload(h->d_Q, h->Q, h->stream));
    DBuf dcnt;
    PG_CUDA(dcnt.ensure(sizeof(unsigned long long) * 64));
    PG_CUDA(cudaMemsetAsync(dcnt.p, 0, sizeof(unsigned long long) * 64, h->stream));
    std::vector<ClassWork> all;
    for (int cu = 0; cu < 10; ++cu)
        for (int cv = 0; cv <= cu; ++cv) {
            const int u0 = h->class_begin[cu], u1 = h->class_begin[cu + 1];
            const int v0 = h->class_begin[cv], v1 = h->class_begin[cv + 1];
            if (u0 == u1 || v0 == v1) continue;
            ClassWork w;
            class_ls(cu, w.la, w.lb);
            class_ls(cv, w.lc, w.ld);
            w.u0 = u0; w.nu = u1 - u0; w.v0 = v0; w.nv = v1 - v0; w.same = cu == cv;
            w.total = w.same ? (long long)w.nu * (w.nu + 1) / 2 : (long long)w.nu * w.nv;
            w.items = w.total > h->rank ? (w.total - h->rank + h->nranks - 1) / h->nranks : 0;
            w.offset = (long long)all.size();
            unscreened += w.total;
            if (w.items) all.push_back(w);
        }
    if (all.size() > 64) return fail(PATGPU_ESTATE, "too many classes");
    for (size_t k = 0; k < all.size(); ++k) {
        EriArgs a = class_args(h, all[k], MODE_RHF, h->tau > 0.0 ? h->tau : -1.0, INFINITY);
        long long blocks = std::min<long long>((a.nquart + 255) / 256, (long long)h->num_sms * 16);
        count_kernel<<<(unsigned)std::max<long long>(blocks, 1), 256, 0, h->stream>>>(
            a, dcnt.as<unsigned long long>() + k);
    }
    PG_CUDA(cudaGetLastError());
    std::vector<unsigned long long> cnt(64, 0);
    PG_CUDA(cudaMemcpyAsync(cnt.data(), dcnt.p, sizeof(unsigned long long) * 64, cudaMemcpyDeviceToHost, h->stream));
    PG_CUDA(cudaStreamSynchronize(h->stream));
    for (size_t k = 0; k < all.size(); ++k) {
        all[k].count = (long long)cnt[k];
        owned += all[k].count;
        if (all[k].count) h->work.push_back(all[k]);
    }
    for (size_t k = 0; k < h->work.size(); ++k) h->work[k].idx = (int)k;
    h->nquart = owned;
    h->nquart_unscreened = unscreened;
    return build_lists(h);
}

// Kernel-variant autotuner: every class has the lane team kernel (0) and the
// shared-memory team kernel (2); the small classes also have the
// register-only kernel (1), the classes whose shared memory leaves room
// for 3 or more blocks an SM the occupancy-hinted shared-memory kernel (5),
// and, on one-primitive handles, every class with at most 32 components on
// one side the warp-synchronous kernel (6).
// Each variant is timed on the first kTuneItems work items of the class's
// own quartet space and the fastest kept.  Runs once per quartet partition,
// on a zero density and the handle's own accumulator (the results are
// discarded).  PATGPU_VARIANT=lane|reg|smem|smem_occ|warp forces a choice where
// it exists.
static int ensure_work(patgpu_basis *h, bool two);

constexpr long long kTuneItems = 1 << 18;

// The tuner's choices are kept for the whole process, per device, class,
// primitive structure (one primitive pair per shell pair or not) and size
// (fewer or more than 8192 quartets): later handles reuse them instead of
// timing again.  Besides saving the tuning of every molecule of a batch,
// this makes the kernel, hence the bits of every quartet's contribution,
// the same in every handle of a process, so that fixed-point builds agree
// bitwise across quartet partitions.
static std::mutex g_tune_lock;
static std::map<std::tuple<int, int, int, int, int>, int> g_tune_cache;

static std::tuple<int, int, int, int, int> tune_key(const patgpu_basis *h, const ClassWork &w, int kind)
{
    return std::make_tuple(h->dev, ((w.la * 4 + w.lb) * 4 + w.lc) * 4 + w.ld, h->single_prim ? 1 : 0,
                           w.count >= 8192 ? 1 : 0, kind);
}

// PATGPU_TUNE_SAVE=<file> appends every choice the tuner makes to <file>;
// PATGPU_TUNE_LOAD=<file> seeds the process's choices from such a file
// before the first tuning, so that a second run (a profiler's, whose own
// launch overhead would distort the timings) launches the same kernels as
// the run that wrote it.  Lines: device class primitive-structure size kind
// variant.
static bool g_tune_loaded = false;

static void tune_load_locked()
{
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char *path = getenv("PATGPU_TUNE_LOAD");
    if (!path) return;
    FILE *f = fopen(path, "r");
    if (!f) return;
    int d, c, sp, big, kind, var;
    while (fscanf(f, "%d %d %d %d %d %d", &d, &c, &sp, &big, &kind, &var) == 6)
        g_tune_cache[std::make_tuple(d, c, sp, big, kind)] = var;
    fclose(f);
}

static bool tune_cached(const patgpu_basis *h, const ClassWork &w, int kind, int *variant)
{
    std::lock_guard<std::mutex> g(g_tune_lock);
    tune_load_locked();
    auto it = g_tune_cache.find(tune_key(h, w, kind));
    if (it == g_tune_cache.end()) return false;
    *variant = it->second;
    return true;
}

static void tune_store(const patgpu_basis *h, const ClassWork &w, int kind, int variant)
{
    std::lock_guard<std::mutex> g(g_tune_lock);
    const auto key = tune_key(h, w, kind);
    g_tune_cache[key] = variant;
    if (const char *path = getenv("PATGPU_TUNE_SAVE")) {
        if (FILE *f = fopen(path, "a")) {
            fprintf(f, "%d %d %d %d %d %d\n", std::get<0>(key), std::get<1>(key), std::get<2>(key), std::get<3>(key),
                    std::get<4>(key), variant);
            fclose(f);
        }
    }
}

static int tune_variants(patgpu_basis *h)
{
    const char *force = getenv("PATGPU_VARIANT");
    int forced = -1;
    if (force && !strcmp(force, "lane")) forced = 0;
    if (force && !strcmp(force, "reg")) forced = 1;
    if (force && !strcmp(force, "smem")) forced = 2;
    if (force && !strcmp(force, "smem_occ")) forced = 5;
    if (force && !strcmp(force, "warp")) forced = h->single_prim ? 6 : -1;
    for (auto &w : h->work) w.variant = 0;
    if (h->work.empty()) return 0;
    if (forced >= 0) {
        for (auto &w : h->work)
            if (eri_has_variant(w.la, w.lb, w.lc, w.ld, forced)) w.variant = forced;
        return 0;
    }
    int rc = ensure_work(h, false);
    if (rc) return rc;
    const size_t nn = (size_t)h->n * h->n;
    cudaStream_t s = h->stream;
    PG_CUDA(cudaMemsetAsync(h->d_D0.p, 0, sizeof(double) * nn, s));
    EriArgs a = h->base_args();
    a.mode = MODE_RHF;
    a.D0 = h->d_D0.as<double>();
    a.A0 = h->d_A0.as<double>();
    cudaEvent_t e0, e1;
    PG_CUDA(cudaEventCreate(&e0));
    PG_CUDA(cudaEventCreate(&e1));
    const bool log = getenv("PATGPU_TUNE_LOG") != nullptr;   // per-class timings to stderr
    for (auto &w : h->work) {
        int cached = 0;
        if (tune_cached(h, w, 0, &cached)) {
            w.variant = cached;
            if (log) fprintf(stderr, "patgpu tune (%d%d|%d%d): variant %d (chosen before)\n", w.la, w.lb, w.lc,
                             w.ld, cached);
            continue;
        }
        a = h->lists ? list_args(h, w, MODE_RHF, 0) : class_args(h, w, MODE_RHF, h->tau > 0.0 ? h->tau : -1.0, INFINITY);
        a.D0 = h->d_D0.as<double>();
        a.A0 = h->d_A0.as<double>();
        a.nquart = std::min(a.nquart, kTuneItems);
        float best = 1e30f;
        for (int var : {0, 1, 2, 5, 6}) {
            if (!eri_has_variant(w.la, w.lb, w.lc, w.ld, var)) continue;
            if (var == 6 && !h->single_prim) continue;
            float ms = 0.f;
            for (int rep = 0; rep < 2; ++rep) {   // first launch warms up
                PG_CUDA(cudaEventRecord(e0, s));
                PG_CUDA(launch_eri_class(w.la, w.lb, w.lc, w.ld, a, s, h->num_sms, var));
                PG_CUDA(cudaEventRecord(e1, s));
                PG_CUDA(cudaEventSynchronize(e1));
                PG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            }
            if (log) fprintf(stderr, "patgpu tune (%d%d|%d%d) %lld quartets: variant %d %.1f us\n", w.la, w.lb, w.lc,
                             w.ld, a.nquart, var, 1e3 * ms);
            if (ms < best) {
                best = ms;
                w.variant = var;
            }
        }
        if (log) fprintf(stderr, "patgpu tune (%d%d|%d%d): chose variant %d\n", w.la, w.lb, w.lc, w.ld, w.variant);
        tune_store(h, w, 0, w.variant);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return 0;
}

// Kernel per class for the mixed-precision window: the FP32 shared-memory
// kernel (3), the FP32 lane kernel (4) and the class's own FP64 kernel,
// timed like tune_variants on the first kTuneItems quartets of the window.
// The FP64 kernel keeps the window where it times faster than both FP32
// kernels (in practice small windows, where a launch's fixed cost outweighs
// the FP32 gain); launch_work then runs both windows as one launch, and
// nquart_fp32 counts only the quartets that do run in FP32.
// PATGPU_VARIANT32=smem|lane|warp forces an FP32 kernel for every class.
static int tune_fp32(patgpu_basis *h)
{
    const char *force = getenv("PATGPU_VARIANT32");
    for (auto &w : h->work) w.variant32 = 3;
    if (force && !strcmp(force, "smem")) return 0;
    if (force && !strcmp(force, "lane")) {
        for (auto &w : h->work) w.variant32 = 4;
        return 0;
    }
    if (force && !strcmp(force, "warp")) {
        for (auto &w : h->work)
            if (h->single_prim && eri_has_variant(w.la, w.lb, w.lc, w.ld, 7)) w.variant32 = 7;
        return 0;
    }
    // timed on the FP32 (term-bound) window, or, when only the density-weighted
    // window of difference builds is set, on the class's whole list
    const bool schwarz_window = h->tau_mix > 0.0;
    if (h->work.empty() || !h->lists || (!schwarz_window && h->tau_dens32 <= 0.0)) return 0;
    int rc = ensure_work(h, false);
    if (rc) return rc;
    const size_t nn = (size_t)h->n * h->n;
    cudaStream_t s = h->stream;
    PG_CUDA(cudaMemsetAsync(h->d_D0.p, 0, sizeof(double) * nn, s));
    cudaEvent_t e0, e1;
    PG_CUDA(cudaEventCreate(&e0));
    PG_CUDA(cudaEventCreate(&e1));
    for (auto &w : h->work) {
        EriArgs a = list_args(h, w, MODE_RHF, schwarz_window ? 1 : 2);
        if (a.nquart <= 0) continue;
        int cached = 0;
        if (tune_cached(h, w, schwarz_window ? 1 : 2, &cached)) {
            w.variant32 = cached;
            continue;
        }
        a.D0 = h->d_D0.as<double>();
        a.A0 = h->d_A0.as<double>();
        a.nquart = std::min(a.nquart, kTuneItems);
        float best = 1e30f;
        for (int var : {3, 4, 7, w.variant}) {
            if (var == 7 && !(h->single_prim && eri_has_variant(w.la, w.lb, w.lc, w.ld, 7))) continue;
            float ms = 0.f;
            for (int rep = 0; rep < 2; ++rep) {
                PG_CUDA(cudaEventRecord(e0, s));
                PG_CUDA(launch_eri_class(w.la, w.lb, w.lc, w.ld, a, s, h->num_sms, var));
                PG_CUDA(cudaEventRecord(e1, s));
                PG_CUDA(cudaEventSynchronize(e1));
                PG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            }
            if (ms < best) {
                best = ms;
                w.variant32 = var;
            }
        }
        tune_store(h, w, schwarz_window ? 1 : 2, w.variant32);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->nquart_fp32 = 0;
    for (const auto &w : h->work)
        if (w.variant32 == 3 || w.variant32 == 4 || w.variant32 == 7) h->nquart_fp32 += w.count - w.nhi;
    return 0;
}

// ------------------------------------------------------- small kernels
__global__ void unpack_kernel(const double *__restrict__ pk, double *__restrict__ full, int n)
{
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long tot = (long long)n * n;
    for (; idx < tot; idx += (long long)gridDim.x * blockDim.x) {
        int i = (int)(idx / n), j = (int)(idx % n);
        int r = i > j ? i : j, c = i > j ? j : i;
        full[idx] = pk[(long long)r * (r + 1) / 2 + c];
    }
}

// packed[ij] = A[i][j] + A[j][i] (j <= i).  det: A holds fixed-point
// elements (two 64-bit words each, acc_add); the two are added exactly and
// rounded once, and a set *err (an out-of-range or non-finite contribution)
// gives NaN everywhere.
__global__ void finish_kernel(const double *__restrict__ A, double *__restrict__ pk, int n, int det,
                              const int *__restrict__ err)
{
    long long no2 = (long long)n * (n + 1) / 2;
    const bool bad = det && err && *err;
    const unsigned long long *U = reinterpret_cast<const unsigned long long *>(A);
    for (long long ij = (long long)blockIdx.x * blockDim.x + threadIdx.x; ij < no2;
         ij += (long long)gridDim.x * blockDim.x) {
        // invert ij = i(i+1)/2 + j
        int i = (int)((sqrt(8.0 * (double)ij + 1.0) - 1.0) * 0.5);
        while ((long long)(i + 1) * (i + 2) / 2 <= ij) ++i;
        while ((long long)i * (i + 1) / 2 > ij) --i;
        int j = (int)(ij - (long long)i * (i + 1) / 2);
        if (!det)
            pk[ij] = A[(size_t)i * n + j] + A[(size_t)j * n + i];
        else
            pk[ij] = bad ? __longlong_as_double(0x7ff8000000000000ll)
                         : fix_sum(U + 2 * ((size_t)i * n + j), U + 2 * ((size_t)j * n + i));
    }
}

// Independent FMA chains: 8 per thread, `iters` steps each.
__global__ void fma_probe_kernel(double *out, int iters, double a, double b)
{
    double x0 = threadIdx.x * 1e-9, x1 = x0 + 0.1, x2 = x0 + 0.2, x3 = x0 + 0.3;
    double x4 = x0 + 0.4, x5 = x0 + 0.5, x6 = x0 + 0.6, x7 = x0 + 0.7;
    for (int i = 0; i < iters; ++i) {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    const double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 1234.5678) out[0] = s;   // keeps the chains alive
}

// FP64 matrix instructions (mma.sync m8n8k4, the only FP64 tensor-core form
// sm_100a has; tcgen05.mma has no FP64 kind): 8 independent accumulator
// pairs per thread, `iters` steps each, 512 flops per warp instruction.
__global__ void dmma_probe_kernel(double *out, int iters, double a, double b)
{
    double c[8][2];
    for (int k = 0; k < 8; ++k) {
        c[k][0] = threadIdx.x * 1e-9 + k;
        c[k][1] = c[k][0] + 0.5;
    }
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                         : "+d"(c[k][0]), "+d"(c[k][1])
                         : "d"(a), "d"(b));
    }
    double s = 0.0;
    for (int k = 0; k < 8; ++k) s += c[k][0] + c[k][1];
    if (s == 1234.5678) out[0] = s;   // keeps the chains alive
}

static int grid_for(long long work, int num_sms)
{
    long long b = (work + 255) / 256;
    long long cap = (long long)num_sms * 8;
    return (int)std::max<long long>(1, std::min(b, cap));
}

// The class launches of one build; timing starts here unless the caller
// recorded ev0 already (a density-screened build times its filter too).
static int launch_fock(patgpu_basis *h, int mode, cudaStream_t s, bool timed_before = false)
{
    EriArgs a = h->base_args();
    a.mode = mode;
    a.D0 = h->d_D0.as<double>();
    a.D1 = h->d_D1.as<double>();
    a.A0 = h->d_A0.as<double>();
    a.A1 = h->d_A1.as<double>();
    if (!timed_before) PG_CUDA(cudaEventRecord(h->ev0, s));
    int launches = 0;
    for (auto &w : h->work) {
        PG_CUDA(launch_work(h, w, a, s));
        ++launches;
    }
    PG_CUDA(cudaEventRecord(h->ev1, s));
    h->last_launches = launches;
    return 0;
}

static int ensure_work(patgpu_basis *h, bool two)
{
    const size_t nn = (size_t)h->n * h->n, no2 = (size_t)h->n * (h->n + 1) / 2;
    PG_CUDA(h->d_D0.ensure(sizeof(double) * nn));
    PG_CUDA(h->d_A0.ensure(2 * sizeof(double) * nn));   // room for fixed-point elements
    PG_CUDA(h->d_Pk0.ensure(sizeof(double) * no2));
    PG_CUDA(h->d_Gk0.ensure(sizeof(double) * no2));
    if (two) {
        PG_CUDA(h->d_D1.ensure(sizeof(double) * nn));
        PG_CUDA(h->d_A1.ensure(2 * sizeof(double) * nn));
        PG_CUDA(h->d_Pk1.ensure(sizeof(double) * no2));
        PG_CUDA(h->d_Gk1.ensure(sizeof(double) * no2));
    }
    return 0;
}

// Bytes of one n x n accumulator in the handle's accumulation mode.
static size_t acc_bytes(const patgpu_basis *h)
{
    return (h->det ? 2 : 1) * sizeof(double) * (size_t)h->n * h->n;
}

// Zero an accumulator (and the handle's device error word) on stream s.
static int acc_clear(const patgpu_basis *h, void *A, cudaStream_t s)
{
    PG_CUDA(cudaMemsetAsync(A, 0, acc_bytes(h), s));
    PG_CUDA(cudaMemsetAsync(h->d_err.p, 0, sizeof(int), s));
    return 0;
}

static int finish(const patgpu_basis *h, const double *A, double *G, cudaStream_t s)
{
    const long long no2 = (long long)h->n * (h->n + 1) / 2;
    finish_kernel<<<grid_for(no2, h->num_sms), 256, 0, s>>>(A, G, h->n, h->det, h->d_err.as<int>());
    PG_CUDA(cudaGetLastError());
    return 0;
}

static int record_timing(patgpu_basis *h)
{
    float ms = 0.f;
    PG_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->last_ns = ms * 1e6;
    return 0;
}

// Largest |D_ij| over the component block of every shell pair (both
// densities when D1 is set); shells without components give 0.
__global__ void shell_dmax_kernel(const double *__restrict__ D0, const double *__restrict__ D1, int n,
                                  const int *__restrict__ soff, const int *__restrict__ snst, int nsh,
                                  double *__restrict__ dsh)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nsh * nsh; idx += gridDim.x * blockDim.x) {
        const int s1 = idx / nsh, s2 = idx - (idx / nsh) * nsh;
        double m = 0.0;
        for (int i = 0; i < snst[s1]; ++i)
            for (int j = 0; j < snst[s2]; ++j) {
                const size_t o = (size_t)(soff[s1] + i) * n + soff[s2] + j;
                m = fmax(m, fabs(D0[o]));
                if (D1) m = fmax(m, fabs(D1[o]));
            }
        dsh[idx] = m;
    }
}

// Append the lanes with keep set to out[*cnt ...] (forward) or, with
// backward, to out[-1 - *cnt ...] (growing down from out), with one
// warp-aggregated atomic.
__device__ __forceinline__ void warp_append(bool keep, unsigned long long v, unsigned long long *out,
                                            unsigned long long *cnt, bool backward)
{
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (!m) return;
    const int lane = threadIdx.x & 31, lead = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == lead) base = atomicAdd(cnt, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, lead);
    const unsigned long long k = base + __popc(m & ((1u << lane) - 1u));
    if (keep) {
        if (backward) *(out - 1 - (long long)k) = v;
        else out[k] = v;
    }
}

// Keep the list entries whose contribution bound Q_ab Q_cd max(4|D_ab|,
// 4|D_cd|, |D_ac|, |D_ad|, |D_bc|, |D_bd|) reaches tau (shell-block maxima;
// the factor 4 covers the Coulomb weight).  A kept entry goes to the FP32
// sublist (written downward from end32) when all32 is set (the FP32 window
// of mixed precision) or its density-weighted term bound (term_bound of the
// class lab, lcd times the same density maximum) is below tau32, else to the
// FP64 sublist (upward from out64); counts in cnt[0] and cnt[1].
__global__ void density_filter_kernel(const EriArgs a, const double *__restrict__ dsh, int nsh,
                                      const double *__restrict__ scr, int all32, int lab, int lcd,
                                      unsigned long long *out64, unsigned long long *end32, unsigned long long *cnt)
{
    const double tau = scr[0], tau32 = scr[1];
    for (long long qi0 = (long long)blockIdx.x * blockDim.x; qi0 < a.nquart;
         qi0 += (long long)gridDim.x * blockDim.x) {
        const long long qi = qi0 + threadIdx.x;
        int u = 0, v = 0;
        bool keep = qi < a.nquart && eri_quartet_at(a, qi, u, v);
        bool low = false;
        if (keep) {
            const int sa = a.pr.sa[u], sb = a.pr.sb[u], sc = a.pr.sa[v], sd = a.pr.sb[v];
            const double dj = 4.0 * fmax(dsh[sa * nsh + sb], dsh[sc * nsh + sd]);
            const double dk = fmax(fmax(dsh[sa * nsh + sc], dsh[sa * nsh + sd]), fmax(dsh[sb * nsh + sc], dsh[sb * nsh + sd]));
            const double dm = fmax(dj, dk);
            keep = a.Q[u] * a.Q[v] * dm >= tau;
            low = all32 || (keep && tau32 > 0.0 && term_bound(a, u, v, lab, lcd) * dm < tau32);
        }
        const unsigned long long k = qi < a.nquart ? a.klist[qi] : 0ull;
        warp_append(keep && !low, k, out64, cnt, false);
        warp_append(keep && low, k, end32, cnt + 1, true);
    }
}

// Filter every class's list(s) against the density of this build (d_D0, and
// d_D1 for UHF) into d_flist, enqueued on s, at the thresholds scr[0] (tau)
// and scr[1] (tau32) in device memory: the counts stay on the device (the
// class launches read them there), so a build with the filter can be
// captured in a CUDA graph, and its thresholds changed between replays.
static int density_filter_enqueue(patgpu_basis *h, bool two, cudaStream_t s, const double *scr)
{
    const int nsh = h->nsh;
    shell_dmax_kernel<<<grid_for((long long)nsh * nsh, h->num_sms), 256, 0, s>>>(
        h->d_D0.as<double>(), two ? h->d_D1.as<double>() : nullptr, h->n, h->d_soff.as<int>(), h->d_snst.as<int>(),
        nsh, h->d_dsh.as<double>());
    const size_t nc = 2 * std::max<size_t>(h->work.size(), 1);
    PG_CUDA(cudaMemsetAsync(h->d_fcnt.p, 0, sizeof(unsigned long long) * nc, s));
    const double lo = h->tau > 0.0 ? h->tau : -1.0;
    const bool mixed = h->tau_mix > lo && h->tau_mix > 0.0;
    unsigned long long *out = h->d_flist.as<unsigned long long>();
    for (const auto &w : h->work)
        for (int win = 0; win < (mixed ? 2 : 1); ++win) {
            EriArgs a = list_args(h, w, MODE_RHF, win);
            if (a.nquart <= 0) continue;
            const int g = (int)std::min<long long>((a.nquart + 255) / 256, (long long)h->num_sms * 16);
            density_filter_kernel<<<std::max(g, 1), 256, 0, s>>>(
                a, h->d_dsh.as<double>(), nsh, scr, win, w.la + w.lb, w.lc + w.ld, out + w.loff,
                out + w.loff + w.count, h->d_fcnt.as<unsigned long long>() + 2 * w.idx);
        }
    PG_CUDA(cudaGetLastError());
    return 0;
}

// Device buffers of the density filter (shell offsets, block maxima, the
// filtered list and its counts).
static int density_filter_buffers(patgpu_basis *h)
{
    if (!h->d_soff.p) {
        std::vector<int> soff(h->nsh), snst(h->nsh);
        for (int i = 0; i < h->nsh; ++i) {
            soff[i] = h->off[i];
            snst[i] = h->nst[i];
        }
        PG_CUDA(upload(h->d_soff, soff, h->stream));
        PG_CUDA(upload(h->d_snst, snst, h->stream));
    }
    PG_CUDA(h->d_dsh.ensure(sizeof(double) * (size_t)h->nsh * h->nsh));
    PG_CUDA(h->d_flist.ensure(std::max<size_t>(h->d_list.bytes, 16)));
    PG_CUDA(h->d_fcnt.ensure(sizeof(unsigned long long) * 2 * std::max<size_t>(h->work.size(), 1)));
    PG_CUDA(h->d_scr.ensure(2 * sizeof(double)));
    return 0;
}

// Calls on a handle must run with the handle's device current: its buffers
// and tables live there.
static int check_device(const patgpu_basis *h)
{
    int d = -1;
    cudaGetDevice(&d);
    if (d != h->dev)
        return fail(PATGPU_ESTATE, "handle built on device %d used with device %d current", h->dev, d);
    return 0;
}

// Host-buffer Fock build shared by the RHF / UHF / JK entry points.
static int host_fock(patgpu_basis *h, int mode, const double *P0, const double *P1, double *G0, double *G1)
{
    if (!h) return fail(PATGPU_EINVAL, "null handle");
    if (int rc0 = check_device(h)) return rc0;
    const bool two = mode != MODE_RHF;
    int rc = ensure_work(h, two);
    if (rc) return rc;
    const size_t nn = (size_t)h->n * h->n, no2 = (size_t)h->n * (h->n + 1) / 2;
    cudaStream_t s = h->stream;
    const int g = grid_for((long long)nn, h->num_sms);
    PG_CUDA(cudaMemcpyAsync(h->d_Pk0.p, P0, sizeof(double) * no2, cudaMemcpyHostToDevice, s));
    unpack_kernel<<<g, 256, 0, s>>>(h->d_Pk0.as<double>(), h->d_D0.as<double>(), h->n);
    if (mode == MODE_UHF) {
        PG_CUDA(cudaMemcpyAsync(h->d_Pk1.p, P1, sizeof(double) * no2, cudaMemcpyHostToDevice, s));
        unpack_kernel<<<g, 256, 0, s>>>(h->d_Pk1.as<double>(), h->d_D1.as<double>(), h->n);
    }
    if ((rc = acc_clear(h, h->d_A0.p, s))) return rc;
    if (two && (rc = acc_clear(h, h->d_A1.p, s))) return rc;
    h->last_computed = h->nquart;
    const bool filt = h->tau_dens > 0.0 && h->lists;
    if (filt) {
        if ((rc = density_filter_buffers(h))) return rc;
        const double scr[2] = {h->tau_dens, h->tau_dens32};   // pageable: staged before the call returns
        PG_CUDA(cudaMemcpyAsync(h->d_scr.p, scr, sizeof(scr), cudaMemcpyHostToDevice, s));
        PG_CUDA(cudaEventRecord(h->ev0, s));
        if ((rc = density_filter_enqueue(h, mode == MODE_UHF, s, h->d_scr.as<double>()))) return rc;
        h->filtered = true;
        h->fcnt.assign(2 * std::max<size_t>(h->work.size(), 1), 0);
    }
    rc = launch_fock(h, mode, s, filt);
    h->filtered = false;
    if (rc) return rc;
    if (filt)
        PG_CUDA(cudaMemcpyAsync(h->fcnt.data(), h->d_fcnt.p, sizeof(unsigned long long) * h->fcnt.size(),
                                cudaMemcpyDeviceToHost, s));
    if ((rc = finish(h, h->d_A0.as<double>(), h->d_Gk0.as<double>(), s))) return rc;
    if (two && (rc = finish(h, h->d_A1.as<double>(), h->d_Gk1.as<double>(), s))) return rc;
    h->h_stage.resize(2 * no2);
    PG_CUDA(cudaMemcpyAsync(h->h_stage.data(), h->d_Gk0.p, sizeof(double) * no2, cudaMemcpyDeviceToHost, s));
    if (two)
        PG_CUDA(cudaMemcpyAsync(h->h_stage.data() + no2, h->d_Gk1.p, sizeof(double) * no2, cudaMemcpyDeviceToHost,
                                s));
    PG_CUDA(cudaStreamSynchronize(s));
    rc = record_timing(h);
    if (rc) return rc;
    if (filt) {
        long long tot = 0;
        for (auto c : h->fcnt) tot += (long long)c;
        h->last_computed = tot;
    }
    for (size_t i = 0; i < no2; ++i) G0[i] += h->h_stage[i];
    if (two)
        for (size_t i = 0; i < no2; ++i) G1[i] += h->h_stage[no2 + i];
    return 0;
}

// Two-electron gradient part: packed half density P, grad[3 ncen] += .
static int grad_2e(patgpu_basis *h, const double *P, const double *PB, double *grad)
{
    if (int rc0 = check_device(h)) return rc0;
    int rc = ensure_work(h, PB != nullptr);
    if (rc) return rc;
    const size_t nn = (size_t)h->n * h->n, no2 = (size_t)h->n * (h->n + 1) / 2;
    cudaStream_t s = h->stream;
    PG_CUDA(cudaMemcpyAsync(h->d_Pk0.p, P, sizeof(double) * no2, cudaMemcpyHostToDevice, s));
    unpack_kernel<<<grid_for((long long)nn, h->num_sms), 256, 0, s>>>(h->d_Pk0.as<double>(), h->d_D0.as<double>(),
                                                                    h->n);
    if (PB) {
        PG_CUDA(cudaMemcpyAsync(h->d_Pk1.p, PB, sizeof(double) * no2, cudaMemcpyHostToDevice, s));
        unpack_kernel<<<grid_for((long long)nn, h->num_sms), 256, 0, s>>>(h->d_Pk1.as<double>(),
                                                                        h->d_D1.as<double>(), h->n);
    }
    DBuf dg;
    const size_t ng = 3 * (size_t)h->ncen;
    PG_CUDA(dg.ensure(sizeof(double) * ng));
    PG_CUDA(cudaMemsetAsync(dg.p, 0, sizeof(double) * ng, s));
    GradArgs ga{};
    ga.ca = h->d_pca.as<int>();
    ga.cb = h->d_pcb.as<int>();
    ga.ea = h->d_pp_ea.as<double>();
    ga.grad = dg.as<double>();
    for (const auto &w : h->work) {
        EriArgs a = h->lists ? list_args(h, w, MODE_RHF, 2)
                             : class_args(h, w, MODE_RHF, h->tau > 0.0 ? h->tau : -1.0, INFINITY);
        a.D0 = h->d_D0.as<double>();
        a.D1 = PB ? h->d_D1.as<double>() : nullptr;
        ga.la = w.la;
        ga.lb = w.lb;
        ga.lc = w.lc;
        ga.ld = w.ld;
        PG_CUDA(launch_eri_grad(a, ga, s, h->num_sms));
    }
    std::vector<double> hg(ng);
    PG_CUDA(cudaMemcpyAsync(hg.data(), dg.p, sizeof(double) * ng, cudaMemcpyDeviceToHost, s));
    PG_CUDA(cudaStreamSynchronize(s));
    for (size_t k = 0; k < ng; ++k) grad[k] += hg[k];
    return 0;
}

// Nuclear repulsion over centre pairs with a non-zero charge product (the
// rule the energy uses; a ghost centre may coincide with the positron).
static void grad_nuc(const patgpu_basis *h, double *grad)
{
    for (int i = 0; i < h->ncen; ++i)
        for (int j = 0; j < i; ++j) {
            const double qq = h->q[i] * h->q[j];
            if (qq == 0.0) continue;
            const double d[3] = {h->xyz[3 * i] - h->xyz[3 * j], h->xyz[3 * i + 1] - h->xyz[3 * j + 1],
                                 h->xyz[3 * i + 2] - h->xyz[3 * j + 2]};
            const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            const double f = qq / (r2 * std::sqrt(r2));
            for (int k = 0; k < 3; ++k) {
                grad[3 * i + k] -= f * d[k];
                grad[3 * j + k] += f * d[k];
            }
        }
}

}  // namespace pg

using namespace pg;

// =================================================================== C ABI
extern "C" {

int patgpu_last_error(void) { return pg::t_err; }
const char *patgpu_error_message(void) { return pg::t_msg; }

int patgpu_rys_host(int n, double T, double *x, double *w)
{
    if (n < 1 || n > RYS_NMAX || !(T >= 0.0) || !x || !w) return fail(PATGPU_EINVAL, "bad Rys request");
    static RysConst rc = host_rys_const();
    for (int f = 0; f < n; ++f) {
        x[f] = rys_eval(n, f, T, rc, rys_coef_host, RYS_DEG);
        w[f] = rys_eval(n, n + f, T, rc, rys_coef_host, RYS_DEG);
    }
    return 0;
}

int patgpu_basis_create(int nshell, const int *l, const int *cen, const int *off, const int *nst,
                        const int *prim_off, const double *alpha, const double *coef, int ncen,
                        const double *charge, const double *xyz, int skipcen, double schwarz_tau,
                        patgpu_handle *out)
{
    return patgpu_basis_create_quartets(nshell, l, cen, off, nst, prim_off, alpha, coef, ncen, charge, xyz, skipcen,
                                        schwarz_tau, 0, 0, 1, out);
}

int patgpu_basis_create_quartets(int nshell, const int *l, const int *cen, const int *off, const int *nst,
                                 const int *prim_off, const double *alpha, const double *coef, int ncen,
                                 const double *charge, const double *xyz, int skipcen, double schwarz_tau,
                                 int start_shell, int rank, int nranks, patgpu_handle *out)
{
    if (nranks < 1 || rank < 0 || rank >= nranks) return fail(PATGPU_EINVAL, "bad partition");
    if (!out || nshell < 1 || ncen < 1 || !l || !cen || !off || !nst || !prim_off || !alpha || !coef || !charge ||
        !xyz)
        return fail(PATGPU_EINVAL, "patgpu_basis_create: null or empty argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        return fail(PATGPU_ENODEV, "no CUDA device: the GPU library has no CPU path");
    int n = 0;
    for (int s = 0; s < nshell; ++s) {
        if (nst[s] && (l[s] < 0 || l[s] > PG_LMAX))
            return fail(PATGPU_EUNSUPPORTED, "shell %d has l = %d; the kernels support l <= %d", s, l[s], PG_LMAX);
        if (nst[s] && nst[s] != ncart(l[s])) return fail(PATGPU_EINVAL, "shell %d: nst %d != ncart(%d)", s, nst[s], l[s]);
        if (cen[s] < 0 || cen[s] >= ncen) return fail(PATGPU_EINVAL, "shell %d: bad centre %d", s, cen[s]);
        if (prim_off[s + 1] <= prim_off[s]) return fail(PATGPU_EINVAL, "shell %d has no primitives", s);
        if (nst[s]) n = std::max(n, off[s] + nst[s]);
    }
    if (n < 1) return fail(PATGPU_EINVAL, "basis has no functions");
    int rc = init_tables();
    if (rc) return rc;
    patgpu_basis *h = new patgpu_basis();
    h->nsh = nshell;
    h->ncen = ncen;
    h->n = n;
    h->skipcen = skipcen;
    h->tau = schwarz_tau;
    h->l.assign(l, l + nshell);
    h->cen.assign(cen, cen + nshell);
    h->off.assign(off, off + nshell);
    h->nst.assign(nst, nst + nshell);
    h->poff.assign(prim_off, prim_off + nshell + 1);
    h->al.assign(alpha, alpha + prim_off[nshell]);
    h->co.assign(coef, coef + prim_off[nshell]);
    h->q.assign(charge, charge + ncen);
    h->xyz.assign(xyz, xyz + 3 * ncen);
    if (const char *e = getenv("PATGPU_DETERMINISTIC")) h->det = strcmp(e, "0") ? 1 : 0;
    int dev = 0;
    cudaGetDevice(&dev);
    h->dev = dev;
    cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess ||
        h->d_err.ensure(sizeof(int)) != cudaSuccess) {
        delete h;
        return fail(PATGPU_ECUDA, "stream/event creation failed");
    }
    cudaMemset(h->d_err.p, 0, sizeof(int));
    h->start_shell = start_shell;
    h->rank = rank;
    h->nranks = nranks;
    rc = build_pairs(h);
    if (!rc) rc = build_schwarz(h);
    if (!rc) rc = build_quartets(h);
    if (!rc) rc = tune_variants(h);
    if (rc) {
        patgpu_basis_destroy(h);
        return rc;
    }
    *out = h;
    return 0;
}

int patgpu_basis_destroy(patgpu_handle h)
{
    if (!h) return 0;
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return 0;
}

int patgpu_set_quartets(patgpu_handle h, int start_shell, int rank, int nranks)
{
    if (!h || nranks < 1 || rank < 0 || rank >= nranks) return fail(PATGPU_EINVAL, "bad partition");
    if (int rc0 = check_device(h)) return rc0;
    h->start_shell = start_shell;
    h->rank = rank;
    h->nranks = nranks;
    int rc = build_quartets(h);
    if (!rc) rc = tune_variants(h);
    // a mixed-precision window set before: count it and tune its kernels
    // again over the new partition
    if (!rc && h->tau_mix > 0.0) rc = patgpu_set_mixed_precision(h, h->tau_mix);
    return rc;
}

int patgpu_rhf_gmatrix(patgpu_handle h, const double *P, double *G)
{
    if (!P || !G) return fail(PATGPU_EINVAL, "null matrix");
    return host_fock(h, MODE_RHF, P, nullptr, G, nullptr);
}

int patgpu_uhf_gmatrix(patgpu_handle h, const double *PA, const double *PB, double *GA, double *GB)
{
    if (!PA || !PB || !GA || !GB) return fail(PATGPU_EINVAL, "null matrix");
    return host_fock(h, MODE_UHF, PA, PB, GA, GB);
}

int patgpu_jk(patgpu_handle h, const double *P, double *J, double *K)
{
    if (!P || !J || !K) return fail(PATGPU_EINVAL, "null matrix");
    return host_fock(h, MODE_JK, P, nullptr, J, K);
}

int patgpu_rhf_accumulate_device(patgpu_handle h, const double *dP, double *dA, void *stream)
{
    if (!h || !dP || !dA) return fail(PATGPU_EINVAL, "null argument");
    if (int rc0 = check_device(h)) return rc0;
    int rc = ensure_work(h, false);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nn = (size_t)h->n * h->n;
    unpack_kernel<<<grid_for((long long)nn, h->num_sms), 256, 0, s>>>(dP, h->d_D0.as<double>(), h->n);
    if ((rc = acc_clear(h, dA, s))) return rc;
    EriArgs a = h->base_args();
    a.mode = MODE_RHF;
    a.D0 = h->d_D0.as<double>();
    a.A0 = dA;
    PG_CUDA(cudaEventRecord(h->ev0, s));
    int launches = 0;
    for (auto &w : h->work) {
        PG_CUDA(launch_work(h, w, a, s));
        ++launches;
    }
    PG_CUDA(cudaEventRecord(h->ev1, s));
    h->last_launches = launches;
    return 0;
}

int patgpu_finish_gmatrix_device(patgpu_handle h, const double *dA, double *dG, void *stream)
{
    if (!h || !dA || !dG) return fail(PATGPU_EINVAL, "null argument");
    if (int rc0 = check_device(h)) return rc0;
    return finish(h, dA, dG, (cudaStream_t)stream);
}

int patgpu_rhf_gmatrix_device(patgpu_handle h, const double *dP, double *dG, void *stream)
{
    if (!h) return fail(PATGPU_EINVAL, "null handle");
    int rc = ensure_work(h, false);
    if (rc) return rc;
    rc = patgpu_rhf_accumulate_device(h, dP, h->d_A0.as<double>(), stream);
    if (rc) return rc;
    return patgpu_finish_gmatrix_device(h, h->d_A0.as<double>(), dG, stream);
}

// ------------------------------------------------ allocation-free build
// patgpu_rhf_gmatrix_device_noalloc keeps its working matrices (the full
// density, n*n doubles, and the unsymmetrised accumulator, n*n elements of
// 16 bytes in the fixed-point mode) in this fixed array instead of buffers
// obtained from cudaMalloc.  It is sized for n <= kNoAllocMaxN basis
// functions: 3 * 512 * 512 doubles = 6 MiB, held by every GPU that loads the
// library until the process exits.  Host code may
// not use the array's name as a device address; the address is looked up
// per device with cudaGetSymbolAddress the first time the entry point runs
// on that device.
}  // extern "C"
namespace pg {
constexpr int kNoAllocMaxN = 512;
static __device__ __align__(256) double g_noalloc_scratch[3 * kNoAllocMaxN * kNoAllocMaxN];
constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_lock;
static double *g_noalloc_ptr[kNoAllocMaxDevices];

static int noalloc_scratch(double **out)
{
    int dev = 0;
    PG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return fail(PATGPU_EINVAL, "device %d is beyond the %d devices the fixed scratch tracks", dev,
                    kNoAllocMaxDevices);
    std::lock_guard<std::mutex> g(g_noalloc_lock);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(PATGPU_ECUDA, "cudaGetSymbolAddress of the fixed scratch failed on device %d: %s", dev,
                        cudaGetErrorString(e));
        g_noalloc_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return 0;
}
}  // namespace pg
extern "C" {

int patgpu_rhf_gmatrix_device_noalloc(patgpu_handle h, const double *dP, double *dG, void *stream)
{
    if (!h || !dP || !dG) return fail(PATGPU_EINVAL, "null argument");
    if (int rc0 = check_device(h)) return rc0;
    if (h->n > kNoAllocMaxN)
        return fail(PATGPU_EINVAL,
                    "patgpu_rhf_gmatrix_device_noalloc: the basis has %d functions but its fixed scratch holds "
                    "at most %d; use patgpu_rhf_gmatrix_device",
                    h->n, kNoAllocMaxN);
    double *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    const int n = h->n;
    const size_t nn = (size_t)n * n;
    double *D = scratch, *A = scratch + nn;
    cudaStream_t s = (cudaStream_t)stream;
    // D is fully rewritten; A keeps the previous call's sums and must start at zero
    unpack_kernel<<<grid_for((long long)nn, h->num_sms), 256, 0, s>>>(dP, D, n);
    PG_CUDA(cudaGetLastError());
    if ((rc = acc_clear(h, A, s))) return rc;
    EriArgs a = h->base_args();
    a.mode = MODE_RHF;
    a.D0 = D;
    a.A0 = A;
    for (auto &w : h->work) {
        PG_CUDA(launch_work(h, w, a, s));
    }
    return finish(h, A, dG, s);
}

int patgpu_eri_quartets(patgpu_handle h, int nq, const int *sh4, double *out)
{
    if (!h || nq < 0 || (nq && (!sh4 || !out))) return fail(PATGPU_EINVAL, "bad arguments");
    if (int rc0 = check_device(h)) return rc0;
    // (shell i, shell j) -> pair index
    std::vector<int> pidx((size_t)h->nsh * h->nsh, -1);
    for (int u = 0; u < h->npair; ++u) {
        pidx[(size_t)h->psa[u] * h->nsh + h->psb[u]] = u;
        pidx[(size_t)h->psb[u] * h->nsh + h->psa[u]] = u;
    }
    std::vector<int2> qs(nq);
    std::vector<char> swapbk(nq);
    for (int k = 0; k < nq; ++k) {
        const int *s = sh4 + 4 * k;
        for (int t = 0; t < 4; ++t)
            if (s[t] < 0 || s[t] >= h->nsh || !h->nst[s[t]]) return fail(PATGPU_EINVAL, "quartet %d: bad shell", k);
        int u = pidx[(size_t)s[0] * h->nsh + s[1]], v = pidx[(size_t)s[2] * h->nsh + s[3]];
        swapbk[k] = h->pcls[u] < h->pcls[v] || (h->pcls[u] == h->pcls[v] && u < v);
        qs[k] = swapbk[k] ? make_int2(v, u) : make_int2(u, v);
    }
    std::vector<double> buf;
    std::vector<long long> offs;
    int rc = export_pairs(h, qs, buf, offs);
    if (rc) return rc;
    size_t o = 0;
    for (int k = 0; k < nq; ++k) {
        const int *s = sh4 + 4 * k;
        const int n0 = h->nst[s[0]], n1 = h->nst[s[1]], n2 = h->nst[s[2]], n3 = h->nst[s[3]];
        // kernel orientation: bra pair (x,y) with x the first shell of the pair
        const int u = qs[k].x, v = qs[k].y;
        const int bx = h->psa[u], kx = h->psa[v];
        const int nby = h->nst[h->psb[u]];
        const int nkx = h->nst[h->psa[v]], nky = h->nst[h->psb[v]];
        const double *blk = buf.data() + offs[k];
        for (int i0 = 0; i0 < n0; ++i0)
            for (int i1 = 0; i1 < n1; ++i1)
                for (int i2 = 0; i2 < n2; ++i2)
                    for (int i3 = 0; i3 < n3; ++i3) {
                        // requested (s0 s1 | s2 s3); kernel (bx by | kx ky) possibly bra/ket swapped
                        int c01[2] = {i0, i1}, c23[2] = {i2, i3};
                        int *cb = swapbk[k] ? c23 : c01, *ck = swapbk[k] ? c01 : c23;
                        const int *sb = swapbk[k] ? s + 2 : s, *skt = swapbk[k] ? s : s + 2;
                        int ibx = (sb[0] == bx) ? cb[0] : cb[1];
                        int iby = (sb[0] == bx) ? cb[1] : cb[0];
                        int ikx = (skt[0] == kx) ? ck[0] : ck[1];
                        int iky = (skt[0] == kx) ? ck[1] : ck[0];
                        out[o++] = blk[(((size_t)ibx * nby + iby) * nkx + ikx) * nky + iky];
                    }
    }
    return 0;
}

// ------------------------------------------------------------ ERI files
}  // extern "C"
namespace pg {

// One record of the reference's ERI files: the layout of ERINT
// (erifs.h:19-22), a double and four unsigned short function indices,
// 16-byte aligned.
struct ErintRecord {
    double val;
    unsigned short i, j, k, l;
};
static_assert(sizeof(ErintRecord) == 16, "ERINT record layout");

// The reference's file stream of two_electron_ints (twoints.c:188-418),
// with the integrals from the GPU: shell quartets in its loop order
// (ish >= start, jsh <= ish, ksh <= ish, lsh <= ksh), on MPI rank r of nproc
// the quartets q with (q + 1) % nproc == r (the card dealing of
// twoints.c:280-288), inside each quartet the component order and the
// canonical restriction of twoints.c:316-337 (j <= i, k <= i, l <= k, and
// l <= j when i = k), records with |v| > 1e-14 (twoints.c:374-379), and a
// new file once a file holds more than max_records (twoints.c:380-386).
// Quartets whose Schwarz bound is below the handle's threshold are skipped
// only when that threshold is at most 1e-14 (then none of their integrals
// reaches the record threshold).  open_file(f) returns file f for writing.
template <class OpenFile>
static int write_eri_stream(patgpu_basis *h, int start, int rank, int nproc, long long max_records,
                            OpenFile open_file, int max_files, int *numints, int *nfiles)
{
    if (h->n > 65536) return fail(PATGPU_EINVAL, "ERI records hold 16-bit function indices; n = %d", h->n);
    const int nsh = h->nsh;
    std::vector<int> pidx((size_t)nsh * nsh, -1);
    for (int u = 0; u < h->npair; ++u) {
        pidx[(size_t)h->psa[u] * nsh + h->psb[u]] = u;
        pidx[(size_t)h->psb[u] * nsh + h->psa[u]] = u;
    }
    const bool screen = h->tau > 0.0 && h->tau <= 1e-14;
    const double threshold = 1e-14;
    int nf = 0;
    long long fsize = 0;
    FILE *out = open_file(0);
    if (!out) return fail(PATGPU_EINVAL, "cannot create ERI file 0");
    std::vector<int> batch;           // 4 shells per quartet
    std::vector<double> vals;
    long long batch_vals = 0;
    const long long kBatchVals = 1LL << 24;   // 128 MiB of integrals per GPU round trip
    std::vector<ErintRecord> recs;
    int rc = 0;
    auto flush = [&]() -> int {
        const int nq = (int)(batch.size() / 4);
        if (!nq) return 0;
        vals.resize((size_t)batch_vals);
        int r = patgpu_eri_quartets(h, nq, batch.data(), vals.data());
        if (r) return r;
        size_t o = 0;
        for (int q = 0; q < nq; ++q) {
            const int *sq = batch.data() + 4 * q;
            const int n0 = h->nst[sq[0]], n1 = h->nst[sq[1]], n2 = h->nst[sq[2]], n3 = h->nst[sq[3]];
            const int o0 = h->off[sq[0]], o1 = h->off[sq[1]], o2 = h->off[sq[2]], o3 = h->off[sq[3]];
            recs.clear();
            for (int a = 0; a < n0; ++a) {
                const int ir = o0 + a;
                for (int b = 0; b < n1; ++b) {
                    const int jr = o1 + b;
                    if (jr > ir) break;
                    for (int c = 0; c < n2; ++c) {
                        const int kr = o2 + c;
                        if (kr > ir) break;
                        for (int d = 0; d < n3; ++d) {
                            const int lr = o3 + d;
                            if (lr > kr) break;
                            if (ir == kr && lr > jr) break;
                            const double v = vals[o + (((size_t)a * n1 + b) * n2 + c) * n3 + d];
                            if (std::fabs(v) > threshold)
                                recs.push_back({v, (unsigned short)ir, (unsigned short)jr, (unsigned short)kr,
                                                (unsigned short)lr});
                        }
                    }
                }
            }
            o += (size_t)n0 * n1 * n2 * n3;
            if (!recs.empty() && std::fwrite(recs.data(), sizeof(ErintRecord), recs.size(), out) != recs.size())
                return fail(PATGPU_EINVAL, "writing ERI file %d failed", nf);
            fsize += (long long)recs.size();
            if (fsize > max_records) {
                std::fclose(out);
                if (nf >= max_files) return fail(PATGPU_EINVAL, "more than %d ERI files", max_files);
                numints[nf++] = (int)fsize;
                out = open_file(nf);
                if (!out) return fail(PATGPU_EINVAL, "cannot create ERI file %d", nf);
                fsize = 0;
            }
        }
        batch.clear();
        batch_vals = 0;
        return 0;
    };
    long long pknt = 0;
    for (int ish = start; ish < nsh && !rc; ++ish)
        for (int jsh = 0; jsh <= ish && !rc; ++jsh)
            for (int ksh = 0; ksh <= ish && !rc; ++ksh)
                for (int lsh = 0; lsh <= ksh && !rc; ++lsh) {
                    ++pknt;
                    if (nproc > 1 && pknt % nproc != rank) continue;
                    if (nproc > 1) pknt = rank;
                    if (!h->nst[ish] || !h->nst[jsh] || !h->nst[ksh] || !h->nst[lsh]) continue;
                    if (screen) {
                        const int u = pidx[(size_t)ish * nsh + jsh], v = pidx[(size_t)ksh * nsh + lsh];
                        if (h->Q[u] * h->Q[v] < h->tau) continue;
                    }
                    batch.insert(batch.end(), {ish, jsh, ksh, lsh});
                    batch_vals += (long long)h->nst[ish] * h->nst[jsh] * h->nst[ksh] * h->nst[lsh];
                    if (batch_vals >= kBatchVals) rc = flush();
                }
    if (!rc) rc = flush();
    if (rc) {
        std::fclose(out);
        return rc;
    }
    std::fclose(out);
    if (fsize) {
        if (nf >= max_files) return fail(PATGPU_EINVAL, "more than %d ERI files", max_files);
        numints[nf++] = (int)fsize;
    }
    *nfiles = nf;
    return 0;
}

}  // namespace pg
extern "C" {

int patgpu_write_eri_files(patgpu_handle h, int start, int rank, int nproc, const char *prefix,
                           const char *basename, long long max_records, int max_files, int *numints, int *nfiles)
{
    if (!h || start < 0 || nproc < 1 || rank < 0 || rank >= nproc || !prefix || !basename || max_records < 1 ||
        max_files < 1 || !numints || !nfiles)
        return fail(PATGPU_EINVAL, "patgpu_write_eri_files: bad argument");
    if (rank > 99999) return fail(PATGPU_EINVAL, "rank too large for the ERI file names");
    const std::string pre(prefix), base(basename);
    auto open_file = [&](int f) -> FILE * {
        if (f > 99999) return nullptr;
        const std::string name = pre + std::to_string(rank) + std::to_string(f) + base;   // erifs.c:54-73
        return std::fopen(name.c_str(), "wb");
    };
    return write_eri_stream(h, start, rank, nproc, max_records, open_file, max_files, numints, nfiles);
}

int patgpu_write_eri_files_with(patgpu_handle h, int start, int rank, int nproc,
                                FILE *(*open_file)(int rank, int file_no, const char *basename),
                                const char *basename, long long max_records, int max_files, int *numints,
                                int *nfiles)
{
    if (!h || start < 0 || nproc < 1 || rank < 0 || rank >= nproc || !open_file || !basename || max_records < 1 ||
        max_files < 1 || !numints || !nfiles)
        return fail(PATGPU_EINVAL, "patgpu_write_eri_files_with: bad argument");
    auto of = [&](int f) -> FILE * { return open_file(rank, f, basename); };
    return write_eri_stream(h, start, rank, nproc, max_records, of, max_files, numints, nfiles);
}

int patgpu_select_device(int index)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return fail(PATGPU_ENODEV, "no CUDA device");
    PG_CUDA(cudaSetDevice(((index % ndev) + ndev) % ndev));
    return 0;
}

int patgpu_fp64_peak(double *tflops)
{
    if (!tflops) return fail(PATGPU_EINVAL, "null argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return fail(PATGPU_ENODEV, "no CUDA device");
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    DBuf out;
    PG_CUDA(out.ensure(sizeof(double)));
    cudaEvent_t e0, e1;
    PG_CUDA(cudaEventCreate(&e0));
    PG_CUDA(cudaEventCreate(&e1));
    const int iters = 1 << 15, threads = 256, blocks = sms * 8;
    fma_probe_kernel<<<blocks, threads>>>(out.as<double>(), iters, 0.999999999, 1e-9);   // warm-up
    PG_CUDA(cudaEventRecord(e0));
    for (int r = 0; r < 4; ++r) fma_probe_kernel<<<blocks, threads>>>(out.as<double>(), iters, 0.999999999, 1e-9);
    PG_CUDA(cudaEventRecord(e1));
    PG_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    PG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *tflops = 4.0 * 2.0 * 8.0 * iters * (double)threads * blocks / (ms * 1e-3) / 1e12;
    return 0;
}

int patgpu_dmma_peak(double *tflops)
{
    if (!tflops) return fail(PATGPU_EINVAL, "null argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return fail(PATGPU_ENODEV, "no CUDA device");
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    DBuf out;
    PG_CUDA(out.ensure(sizeof(double)));
    cudaEvent_t e0, e1;
    PG_CUDA(cudaEventCreate(&e0));
    PG_CUDA(cudaEventCreate(&e1));
    const int iters = 1 << 12, threads = 256, blocks = sms * 8;
    dmma_probe_kernel<<<blocks, threads>>>(out.as<double>(), iters, 0.999999999, 1e-9);   // warm-up
    PG_CUDA(cudaEventRecord(e0));
    for (int r = 0; r < 4; ++r) dmma_probe_kernel<<<blocks, threads>>>(out.as<double>(), iters, 0.999999999, 1e-9);
    PG_CUDA(cudaEventRecord(e1));
    PG_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    PG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double warps = (double)threads / 32.0 * blocks;
    *tflops = 4.0 * 512.0 * 8.0 * iters * warps / (ms * 1e-3) / 1e12;
    return 0;
}

int patgpu_set_deterministic(patgpu_handle h, int on)
{
    if (!h) return fail(PATGPU_EINVAL, "null handle");
    h->det = on ? 1 : 0;
    return 0;
}

int patgpu_accumulator_bytes(patgpu_handle h, size_t *bytes)
{
    if (!h || !bytes) return fail(PATGPU_EINVAL, "null argument");
    *bytes = acc_bytes(h);
    return 0;
}

int patgpu_set_mixed_precision(patgpu_handle h, double tau_fp32)
{
    if (!h || !(tau_fp32 >= 0.0)) return fail(PATGPU_EINVAL, "bad mixed-precision threshold");
    if (int rc0 = check_device(h)) return rc0;
    h->tau_mix = tau_fp32;
    h->nquart_fp32 = 0;
    if (tau_fp32 <= 0.0 || tau_fp32 <= h->tau) return h->lists ? build_lists(h) : 0;
    // the lists split each class by term_bound (build_lists); mixed
    // precision runs over the compacted lists only
    int rc = h->lists ? build_lists(h) : 0;
    if (rc || !h->lists) return rc;
    for (const auto &w : h->work) h->nquart_fp32 += w.count - w.nhi;
    return tune_fp32(h);
}

int patgpu_mixed_stats(patgpu_handle h, long long *n_fp32)
{
    if (!h || !n_fp32) return fail(PATGPU_EINVAL, "null argument");
    *n_fp32 = h->nquart_fp32;
    return 0;
}

int patgpu_stats(patgpu_handle h, long long *o)
{
    if (!h || !o) return fail(PATGPU_EINVAL, "null argument");
    o[0] = h->n;
    o[1] = h->npair;
    o[2] = h->nquart;
    o[3] = (long long)h->work.size();
    o[4] = h->nquart_unscreened;
    return 0;
}

int patgpu_class_counts(patgpu_handle h, int max, int *l4, long long *counts)
{
    if (!h || !l4 || !counts) return fail(PATGPU_EINVAL, "null argument");
    int k = 0;
    for (auto &w : h->work) {
        if (k >= max) break;
        l4[4 * k] = w.la; l4[4 * k + 1] = w.lb; l4[4 * k + 2] = w.lc; l4[4 * k + 3] = w.ld;
        counts[k] = w.count;
        ++k;
    }
    return k;
}

int patgpu_last_timing(patgpu_handle h, double *ns, int *launches)
{
    if (!h) return fail(PATGPU_EINVAL, "null handle");
    if (ns) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, h->ev0, h->ev1) == cudaSuccess) h->last_ns = ms * 1e6;
        *ns = h->last_ns;
    }
    if (launches) *launches = h->last_launches;
    return 0;
}

int patgpu_oneints(patgpu_handle h, double *S, double *T, double *H)
{
    if (!h || !S || !T || !H) return fail(PATGPU_EINVAL, "null argument");
    if (int rc0 = check_device(h)) return rc0;
    return run_oneints(h->nsh, h->l.data(), h->cen.data(), h->off.data(), h->nst.data(), h->poff.data(),
                       h->al.data(), h->co.data(), h->ncen, h->q.data(), h->xyz.data(), h->skipcen, h->n, S, T, H,
                       nullptr, h->stream);
}

int patgpu_onebody(int nshell, const int *l, const int *cen, const int *off, const int *nst,
                   const int *prim_off, const double *alpha, const double *coef, int ncen,
                   const double *charge, const double *xyz, int skipcen, double *S, double *T,
                   double *H, double *Hdpm)
{
    if (nshell < 1 || !l || !cen || !off || !nst || !prim_off || !alpha || !coef || !charge || !xyz)
        return fail(PATGPU_EINVAL, "patgpu_onebody: null argument");
    if ((S || T || H) && !(S && T && H)) return fail(PATGPU_EINVAL, "patgpu_onebody: S, T, H go together");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        return fail(PATGPU_ENODEV, "no CUDA device: the GPU library has no CPU path");
    int n = 0;
    for (int s = 0; s < nshell; ++s) {
        if (nst[s] && (l[s] < 0 || l[s] > PG_LMAX))
            return fail(PATGPU_EUNSUPPORTED, "shell %d has l = %d; the kernels support l <= %d", s, l[s], PG_LMAX);
        if (nst[s]) n = std::max(n, off[s] + nst[s]);
    }
    int rc = init_tables();
    if (rc) return rc;
    return run_oneints(nshell, l, cen, off, nst, prim_off, alpha, coef, ncen, charge, xyz, skipcen, n, S, T, H, Hdpm,
                       nullptr);
}

int patgpu_moments(int nshell, const int *l, const int *cen, const int *off, const int *nst, const int *prim_off,
                   const double *alpha, const double *coef, int ncen, const double *xyz, double *dip, double *quad)
{
    if (nshell < 1 || !l || !cen || !off || !nst || !prim_off || !alpha || !coef || !xyz || !dip || !quad)
        return fail(PATGPU_EINVAL, "patgpu_moments: null argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        return fail(PATGPU_ENODEV, "no CUDA device: the GPU library has no CPU path");
    int n = 0;
    for (int s = 0; s < nshell; ++s) {
        if (nst[s] && (l[s] < 0 || l[s] > PG_LMAX))
            return fail(PATGPU_EUNSUPPORTED, "shell %d has l = %d; the kernels support l <= %d", s, l[s], PG_LMAX);
        if (nst[s]) n = std::max(n, off[s] + nst[s]);
    }
    int rc = init_tables();
    if (rc) return rc;
    return run_moments(nshell, l, cen, off, nst, prim_off, alpha, coef, ncen, xyz, n, dip, quad, nullptr);
}

int patgpu_uhf_gradient(patgpu_handle h, const double *PA, const double *PB, const double *WA, const double *WB,
                        int parts, int with_dpm, double *grad)
{
    if (!h || !PA || !PB || !grad || parts < 0 || parts > PATGPU_GRAD_ALL)
        return fail(PATGPU_EINVAL, "patgpu_uhf_gradient: bad argument");
    if ((parts & PATGPU_GRAD_1E) && (!WA || !WB)) return fail(PATGPU_EINVAL, "patgpu_uhf_gradient: the 1e part needs W");
    const size_t ng = 3 * (size_t)h->ncen, no2 = (size_t)h->n * (h->n + 1) / 2;
    std::fill(grad, grad + ng, 0.0);
    if (parts & PATGPU_GRAD_2E) {
        int rc = grad_2e(h, PA, PB, grad);
        if (rc) return rc;
    }
    if (parts & PATGPU_GRAD_1E) {
        // sum over spins of tr(P_s dH) - tr(W_s dS) = 2 tr(P dH) - 2 tr(W dS)
        // with the closed-shell-like P = (Pa + Pb)/2 and W = (Wa + Wb)/2
        std::vector<double> Ph(no2), Wh(no2), g1(ng, 0.0);
        for (size_t k = 0; k < no2; ++k) {
            Ph[k] = 0.5 * (PA[k] + PB[k]);
            Wh[k] = 0.5 * (WA[k] + WB[k]);
        }
        int rc = run_onebody_grad(h->nsh, h->l.data(), h->cen.data(), h->off.data(), h->nst.data(), h->poff.data(),
                                  h->al.data(), h->co.data(), h->ncen, h->q.data(), h->xyz.data(), h->skipcen, h->n,
                                  Ph.data(), Wh.data(), with_dpm, g1.data(), h->stream);
        if (rc) return rc;
        for (size_t k = 0; k < ng; ++k) grad[k] += g1[k];
    }
    if (parts & PATGPU_GRAD_NUC) grad_nuc(h, grad);
    return 0;
}

int patgpu_set_density_screening(patgpu_handle h, double tau_dens)
{
    if (!h || !(tau_dens >= 0.0)) return fail(PATGPU_EINVAL, "bad density-screening threshold");
    h->tau_dens = tau_dens;
    return 0;
}

int patgpu_set_density_precision(patgpu_handle h, double tau32)
{
    if (!h || !(tau32 >= 0.0)) return fail(PATGPU_EINVAL, "bad density-weighted precision threshold");
    if (int rc0 = check_device(h)) return rc0;
    const bool retune = tau32 > 0.0 && h->tau_dens32 <= 0.0 && h->tau_mix <= 0.0;
    h->tau_dens32 = tau32;
    return retune ? tune_fp32(h) : 0;
}

int patgpu_last_computed(patgpu_handle h, long long *quartets)
{
    if (!h || !quartets) return fail(PATGPU_EINVAL, "null argument");
    *quartets = h->last_computed;
    return 0;
}

int patgpu_rhf_gradient(patgpu_handle h, const double *P, const double *W, int parts, int with_dpm,
                        double *grad)
{
    if (!h || !P || !grad || parts < 0 || parts > PATGPU_GRAD_ALL)
        return fail(PATGPU_EINVAL, "patgpu_rhf_gradient: bad argument");
    if ((parts & PATGPU_GRAD_1E) && !W) return fail(PATGPU_EINVAL, "patgpu_rhf_gradient: the 1e part needs W");
    const size_t ng = 3 * (size_t)h->ncen;
    std::fill(grad, grad + ng, 0.0);
    if (parts & PATGPU_GRAD_2E) {
        int rc = grad_2e(h, P, nullptr, grad);
        if (rc) return rc;
    }
    if (parts & PATGPU_GRAD_1E) {
        std::vector<double> g1(ng, 0.0);
        int rc = run_onebody_grad(h->nsh, h->l.data(), h->cen.data(), h->off.data(), h->nst.data(), h->poff.data(),
                                  h->al.data(), h->co.data(), h->ncen, h->q.data(), h->xyz.data(), h->skipcen, h->n, P,
                                  W, with_dpm, g1.data(), h->stream);
        if (rc) return rc;
        for (size_t k = 0; k < ng; ++k) grad[k] += g1[k];
    }
    if (parts & PATGPU_GRAD_NUC) grad_nuc(h, grad);
    return 0;
}

int patgpu_dpm(patgpu_handle h, double *H)
{
    if (!h || !H) return fail(PATGPU_EINVAL, "null argument");
    if (int rc0 = check_device(h)) return rc0;
    return run_oneints(h->nsh, h->l.data(), h->cen.data(), h->off.data(), h->nst.data(), h->poff.data(),
                       h->al.data(), h->co.data(), h->ncen, h->q.data(), h->xyz.data(), h->skipcen, h->n, nullptr,
                       nullptr, nullptr, H, h->stream);
}


}  // extern "C"

// ================================================================ batches
// Many molecules advanced together: one CUDA graph holds every molecule's
// Fock build (density unpack, accumulator clear, its quartet-class launches
// in class order, the symmetrising finish), spread over up to kBatchStreams
// capture streams so that molecules can run side by side, or kept on one
// (batch_capture times both on the first capture of each graph kind).  The
// graph is captured on the first launch (after one plain warm-up build per
// molecule, which also configures every kernel) and replayed afterwards;
// changing a molecule's mixed-precision threshold drops it.
struct patgpu_batch_s {
    std::vector<patgpu_basis *> mols;
    std::unique_ptr<pg::DBuf[]> dP, dG;   // packed n(n+1)/2 per molecule
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> join;
    cudaStream_t cs = nullptr;
    cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
    // [0]: plain builds; [1]: density-screened builds (incremental SCF),
    // the filter of every molecule inside the graph
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    int nodes[2] = {0, 0};
    // side streams each graph spreads the molecules over (0: not chosen yet)
    int nside[2] = {0, 0};
    int screened = 0;                      // launches use graph [1]
    // the screening thresholds of graph [1], {tau_dens, tau32} per molecule:
    // pinned host pairs that the graph's first node copies to d_scr on
    // every replay, so new thresholds need no new capture
    double *h_scr = nullptr;
    pg::DBuf d_scr;
    double last_ns = 0.0;
    std::vector<double> stage;
};

namespace pg {

constexpr int kBatchStreams = 8;

static void batch_drop_graph(patgpu_batch_s *b, int which = -1)
{
    for (int k = 0; k < 2; ++k) {
        if (which >= 0 && k != which) continue;
        if (b->exec[k]) cudaGraphExecDestroy(b->exec[k]);
        if (b->graph[k]) cudaGraphDestroy(b->graph[k]);
        b->exec[k] = nullptr;
        b->graph[k] = nullptr;
        b->nodes[k] = 0;
    }
}

// One molecule's Fock build on stream s from the batch buffers; screened:
// the density filter of the molecule's handle first, then the class
// launches over its sublists (counts read on the device).
static int batch_enqueue(patgpu_batch_s *b, int m, cudaStream_t s, bool screened)
{
    patgpu_basis *h = b->mols[m];
    const size_t nn = (size_t)h->n * h->n;
    unpack_kernel<<<grid_for((long long)nn, h->num_sms), 256, 0, s>>>(b->dP[m].as<double>(), h->d_D0.as<double>(),
                                                                    h->n);
    if (int rc = acc_clear(h, h->d_A0.p, s)) return rc;
    // graph [1] filters every molecule with lists, at its own thresholds (a
    // threshold of 0 keeps every quartet)
    const bool filt = screened && h->lists;
    if (filt) {
        if (int rc = density_filter_enqueue(h, false, s, b->d_scr.as<double>() + 2 * m)) return rc;
        h->filtered = true;
    }
    EriArgs a = h->base_args();
    a.mode = MODE_RHF;
    a.D0 = h->d_D0.as<double>();
    a.A0 = h->d_A0.as<double>();
    cudaError_t e = cudaSuccess;
    for (const auto &w : h->work)
        if (e == cudaSuccess) e = launch_work(h, w, a, s);
    h->filtered = false;
    PG_CUDA(e);
    return finish(h, h->d_A0.as<double>(), b->dG[m].as<double>(), s);
}

// Capture graph [k] over ns of the side streams into *g / *x.
static int batch_capture_streams(patgpu_batch_s *b, int k, int ns, cudaGraph_t *g, cudaGraphExec_t *x)
{
    const bool screened = k == 1;
    const int nm = (int)b->mols.size();
    const size_t scr_bytes = 2 * sizeof(double) * (size_t)nm;
    // heaviest molecules first, dealt round-robin over the capture streams
    std::vector<int> order(nm);
    for (int m = 0; m < nm; ++m) order[m] = m;
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return b->mols[x]->nquart > b->mols[y]->nquart; });
    PG_CUDA(cudaStreamBeginCapture(b->cs, cudaStreamCaptureModeThreadLocal));
    int rc = 0;
    // graph [1] first copies the current thresholds from the pinned pairs
    cudaError_t e = screened ? cudaMemcpyAsync(b->d_scr.p, b->h_scr, scr_bytes, cudaMemcpyHostToDevice, b->cs)
                             : cudaSuccess;
    if (e == cudaSuccess) e = cudaEventRecord(b->fork, b->cs);
    for (int i = 0; e == cudaSuccess && i < ns; ++i) e = cudaStreamWaitEvent(b->side[i], b->fork, 0);
    for (int i = 0; e == cudaSuccess && !rc && i < nm; ++i) rc = batch_enqueue(b, order[i], b->side[i % ns], screened);
    for (int i = 0; e == cudaSuccess && !rc && i < ns; ++i) {
        e = cudaEventRecord(b->join[i], b->side[i]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->cs, b->join[i], 0);
    }
    *g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(b->cs, g);
    if (rc || e != cudaSuccess || e2 != cudaSuccess) {
        if (*g) cudaGraphDestroy(*g);
        *g = nullptr;
        if (rc) return rc;
        return fail(PATGPU_ECUDA, "batch capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    if (cudaGraphInstantiate(x, *g, 0) != cudaSuccess) {
        cudaGraphDestroy(*g);
        *g = nullptr;
        return fail(PATGPU_ECUDA, "batch graph instantiation failed");
    }
    return 0;
}

// Capture graph [k] (0: plain builds, 1: density-screened builds).  The
// first capture of each kind also chooses how many side streams the
// molecules are spread over: all of them (molecules run side by side and
// fill each other's tails) or one (each launch has the GPU to itself; the
// class kernels' grids already fill every SM once).  Both graphs are timed
// on one launch each over the buffers' current densities and the faster is
// kept, and the choice holds for later captures of that kind.
static int batch_capture(patgpu_batch_s *b, int k)
{
    const bool screened = k == 1;
    const int nm = (int)b->mols.size();
    const size_t scr_bytes = 2 * sizeof(double) * (size_t)nm;
    if (screened) PG_CUDA(cudaMemcpyAsync(b->d_scr.p, b->h_scr, scr_bytes, cudaMemcpyHostToDevice, b->cs));
    // warm-up outside the capture: configures every kernel it will launch
    for (int m = 0; m < nm; ++m) {
        int rc = batch_enqueue(b, m, b->cs, screened);
        if (rc) return rc;
    }
    PG_CUDA(cudaStreamSynchronize(b->cs));
    const int all = (int)b->side.size();
    if (b->nside[k] > 0 || all == 1) {
        const int ns = b->nside[k] > 0 ? b->nside[k] : all;
        if (int rc = batch_capture_streams(b, k, ns, &b->graph[k], &b->exec[k])) return rc;
    } else {
        cudaGraph_t g[2] = {nullptr, nullptr};
        cudaGraphExec_t x[2] = {nullptr, nullptr};
        const int ns[2] = {all, 1};
        float ms[2] = {0.f, 0.f};
        int rc = 0;
        for (int c = 0; c < 2 && !rc; ++c) {
            rc = batch_capture_streams(b, k, ns[c], &g[c], &x[c]);
            if (!rc && (cudaEventRecord(b->ev0, b->cs) != cudaSuccess || cudaGraphLaunch(x[c], b->cs) != cudaSuccess ||
                        cudaEventRecord(b->ev1, b->cs) != cudaSuccess || cudaEventSynchronize(b->ev1) != cudaSuccess ||
                        cudaEventElapsedTime(&ms[c], b->ev0, b->ev1) != cudaSuccess))
                rc = fail(PATGPU_ECUDA, "batch stream-count trial failed");
        }
        const int keep = (!rc && ms[1] < ms[0]) ? 1 : 0;
        for (int c = 0; c < 2; ++c) {
            if (c == keep && !rc) continue;
            if (x[c]) cudaGraphExecDestroy(x[c]);
            if (g[c]) cudaGraphDestroy(g[c]);
        }
        if (rc) return rc;
        b->graph[k] = g[keep];
        b->exec[k] = x[keep];
        b->nside[k] = ns[keep];
    }
    size_t nodes = 0;
    PG_CUDA(cudaGraphGetNodes(b->graph[k], nullptr, &nodes));
    b->nodes[k] = (int)nodes;
    return 0;
}

}  // namespace pg

extern "C" {

int patgpu_batch_create(int nmol, const patgpu_handle *mols, patgpu_batch *out)
{
    if (!out || nmol < 1 || !mols) return fail(PATGPU_EINVAL, "patgpu_batch_create: bad argument");
    *out = nullptr;
    for (int m = 0; m < nmol; ++m) {
        if (!mols[m]) return fail(PATGPU_EINVAL, "patgpu_batch_create: molecule %d has no handle", m);
        if (int rc0 = check_device(mols[m])) return rc0;
    }
    auto *b = new patgpu_batch_s();
    b->mols.assign(mols, mols + nmol);
    b->dP.reset(new DBuf[nmol]);
    b->dG.reset(new DBuf[nmol]);
    auto bad = [&](const char *what) {
        patgpu_batch_destroy(b);
        return fail(PATGPU_ECUDA, "patgpu_batch_create: %s", what);
    };
    for (int m = 0; m < nmol; ++m) {
        patgpu_basis *h = mols[m];
        const size_t no2 = (size_t)h->n * (h->n + 1) / 2;
        if (ensure_work(h, false) || b->dP[m].ensure(sizeof(double) * no2) != cudaSuccess ||
            b->dG[m].ensure(sizeof(double) * no2) != cudaSuccess ||
            cudaMemset(b->dP[m].p, 0, sizeof(double) * no2) != cudaSuccess)
            return bad("device buffers");
    }
    if (cudaMallocHost((void **)&b->h_scr, 2 * sizeof(double) * nmol) != cudaSuccess ||
        b->d_scr.ensure(2 * sizeof(double) * nmol) != cudaSuccess)
        return bad("threshold buffers");
    for (int k = 0; k < 2 * nmol; ++k) b->h_scr[k] = 0.0;
    if (cudaStreamCreateWithFlags(&b->cs, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess)
        return bad("streams/events");
    const int ns = std::min(kBatchStreams, nmol);
    for (int k = 0; k < ns; ++k) {
        cudaStream_t s = nullptr;
        cudaEvent_t ev = nullptr;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return bad("streams");
        b->side.push_back(s);
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return bad("events");
        b->join.push_back(ev);
    }
    *out = b;
    return 0;
}

int patgpu_batch_destroy(patgpu_batch b)
{
    if (!b) return 0;
    if (b->cs) cudaStreamSynchronize(b->cs);
    batch_drop_graph(b);
    for (auto s : b->side) cudaStreamDestroy(s);
    for (auto e : b->join) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->cs) cudaStreamDestroy(b->cs);
    if (b->h_scr) cudaFreeHost(b->h_scr);
    delete b;
    return 0;
}

int patgpu_batch_buffers(patgpu_batch b, int m, double **dP, double **dG)
{
    if (!b || m < 0 || m >= (int)b->mols.size() || !dP || !dG) return fail(PATGPU_EINVAL, "bad batch buffer request");
    *dP = b->dP[m].as<double>();
    *dG = b->dG[m].as<double>();
    return 0;
}

int patgpu_batch_set_mixed_precision(patgpu_batch b, double tau_fp32)
{
    if (!b) return fail(PATGPU_EINVAL, "null batch");
    for (auto *h : b->mols) {
        int rc = patgpu_set_mixed_precision(h, tau_fp32);
        if (rc) return rc;
    }
    batch_drop_graph(b);
    return 0;
}

int patgpu_batch_set_density_thresholds(patgpu_batch b, const double *tau_dens, const double *tau32)
{
    if (!b || !tau_dens) return fail(PATGPU_EINVAL, "patgpu_batch_set_density_thresholds: null argument");
    const int nm = (int)b->mols.size();
    bool any = false, any32 = false;
    for (int m = 0; m < nm; ++m) {
        const double t = tau_dens[m], t32 = tau32 ? tau32[m] : 0.0;
        if (!(t >= 0.0) || !(t32 >= 0.0))
            return fail(PATGPU_EINVAL, "patgpu_batch_set_density_thresholds: bad threshold of molecule %d", m);
        any = any || t > 0.0;
        any32 = any32 || t32 > 0.0;
    }
    b->screened = any ? 1 : 0;
    if (!any) return 0;   // plain graph; graph [1] keeps its structure for later
    // graph [1] reads the thresholds at replay: only a change of its launch
    // structure (first use, or the first tau32 > 0) needs a new capture
    bool recapture = !b->exec[1];
    for (int m = 0; m < nm; ++m) {
        patgpu_basis *h = b->mols[m];
        const double t32 = tau32 ? tau32[m] : 0.0;
        if (any32 && !h->dens32_armed) {
            int rc = patgpu_set_density_precision(h, std::max(t32, 1e-300));
            if (rc) return rc;
            h->dens32_armed = true;
            recapture = true;
        }
        h->tau_dens = tau_dens[m];
        h->tau_dens32 = t32;
        if (h->lists)
            if (int rc = density_filter_buffers(h)) return rc;
        b->h_scr[2 * m] = tau_dens[m];
        b->h_scr[2 * m + 1] = t32;
    }
    if (recapture) batch_drop_graph(b, 1);
    return 0;
}

int patgpu_batch_set_density_screening(patgpu_batch b, double tau_dens, double tau32)
{
    if (!b || !(tau_dens >= 0.0) || !(tau32 >= 0.0)) return fail(PATGPU_EINVAL, "bad batch screening threshold");
    const std::vector<double> t(b->mols.size(), tau_dens), t32(b->mols.size(), tau32);
    return patgpu_batch_set_density_thresholds(b, t.data(), t32.data());
}

int patgpu_batch_last_computed(patgpu_batch b, long long *quartets)
{
    if (!b || !quartets) return fail(PATGPU_EINVAL, "null argument");
    long long tot = 0;
    PG_CUDA(cudaStreamSynchronize(b->cs));
    for (auto *h : b->mols) {
        if (!b->screened || !h->lists) {
            tot += h->nquart;
            continue;
        }
        std::vector<unsigned long long> c(2 * std::max<size_t>(h->work.size(), 1), 0);
        PG_CUDA(cudaMemcpy(c.data(), h->d_fcnt.p, sizeof(unsigned long long) * c.size(), cudaMemcpyDeviceToHost));
        for (auto x : c) tot += (long long)x;
    }
    *quartets = tot;
    return 0;
}

int patgpu_batch_launch(patgpu_batch b, void *stream)
{
    if (!b) return fail(PATGPU_EINVAL, "null batch");
    const int k = b->screened;
    if (!b->exec[k]) {
        int rc = batch_capture(b, k);
        if (rc) return rc;
    }
    cudaStream_t s = (cudaStream_t)stream;
    PG_CUDA(cudaEventRecord(b->ev0, s));
    PG_CUDA(cudaGraphLaunch(b->exec[k], s));
    PG_CUDA(cudaEventRecord(b->ev1, s));
    return 0;
}

int patgpu_batch_rhf_gmatrix(patgpu_batch b, const double *const *P, double *const *G)
{
    if (!b || !P || !G) return fail(PATGPU_EINVAL, "patgpu_batch_rhf_gmatrix: null argument");
    const int nm = (int)b->mols.size();
    size_t tot = 0;
    for (int m = 0; m < nm; ++m) {
        if (!P[m] || !G[m]) return fail(PATGPU_EINVAL, "patgpu_batch_rhf_gmatrix: molecule %d has no matrix", m);
        tot += (size_t)b->mols[m]->n * (b->mols[m]->n + 1) / 2;
    }
    // densities first: a first capture times its graphs over them
    for (int m = 0; m < nm; ++m) {
        const size_t no2 = (size_t)b->mols[m]->n * (b->mols[m]->n + 1) / 2;
        PG_CUDA(cudaMemcpyAsync(b->dP[m].p, P[m], sizeof(double) * no2, cudaMemcpyHostToDevice, b->cs));
    }
    if (!b->exec[b->screened]) {
        int rc = batch_capture(b, b->screened);
        if (rc) return rc;
    }
    int rc = patgpu_batch_launch(b, b->cs);
    if (rc) return rc;
    b->stage.resize(tot);
    size_t o = 0;
    for (int m = 0; m < nm; ++m) {
        const size_t no2 = (size_t)b->mols[m]->n * (b->mols[m]->n + 1) / 2;
        PG_CUDA(cudaMemcpyAsync(b->stage.data() + o, b->dG[m].p, sizeof(double) * no2, cudaMemcpyDeviceToHost, b->cs));
        o += no2;
    }
    PG_CUDA(cudaStreamSynchronize(b->cs));
    o = 0;
    for (int m = 0; m < nm; ++m) {
        const size_t no2 = (size_t)b->mols[m]->n * (b->mols[m]->n + 1) / 2;
        for (size_t k = 0; k < no2; ++k) G[m][k] += b->stage[o + k];
        o += no2;
    }
    return 0;
}

int patgpu_batch_stats(patgpu_batch b, long long *out4)
{
    if (!b || !out4) return fail(PATGPU_EINVAL, "null argument");
    long long q = 0, q32 = 0;
    for (auto *h : b->mols) {
        q += h->nquart;
        q32 += h->nquart_fp32;
    }
    out4[0] = (long long)b->mols.size();
    out4[1] = q;
    out4[2] = q32;
    out4[3] = b->nodes[b->screened] ? b->nodes[b->screened] : b->nodes[0];
    return 0;
}

int patgpu_batch_last_timing(patgpu_batch b, double *ns)
{
    if (!b || !ns) return fail(PATGPU_EINVAL, "null argument");
    float ms = 0.f;
    PG_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    *ns = ms * 1e6;
    return 0;
}

}  // extern "C"
