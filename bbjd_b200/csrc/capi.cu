// C-ABI of libbbjd_gpu.so: the reference's public functions (include/bbjd.h)
// and the device-operator extension (include/bbjd_gpu.h).
#include "engine.cuh"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <thread>
#include <algorithm>
#include <atomic>
#include <mutex>

namespace bbjd {

// ---------------------------------------------------------------------------
// Device operators: fused BBT product, device preconditioner.
struct DeviceOps : Operators {
    const bbjd_bbt_matrix *m;
    const bbjd_precond *pc;
    cudaStream_t st;
    BBTScratch sc;   // this solve's own product scratch
    DeviceOps(const bbjd_bbt_matrix *m_, const bbjd_precond *pc_, cudaStream_t s) : m(m_), pc(pc_), st(s) {}
    ~DeviceOps() override { bbt_scratch_free(&sc); }
    bbjd_status apply(const cplx *x, cplx *yA, cplx *yB, cplx ta, cplx tb, cplx *r,
                      double *rnorm_dev) override {
        return bbt_apply(m, &sc, x, yA, yB, ta, tb, r, rnorm_dev, st);
    }
    bool has_precond() const override { return pc != nullptr; }
    bbjd_status precond(int nrhs, const cplx *r, cplx *x) override {
        return precond_solve(pc, nrhs, r, x, m->n, st);
    }
    double apply_bytes(bool residual) const override { return bbt_bytes(m, residual); }
    double precond_bytes(int nrhs) const override { return pc ? bbjd::precond_bytes(pc, nrhs) : 0.0; }
};

Operators *make_device_ops(const bbjd_bbt_matrix *m, const bbjd_precond *pc, Scratch *,
                           cudaStream_t st) {
    auto *o = new (std::nothrow) DeviceOps(m, pc, st);
    if (o && bbt_scratch_alloc(m, &o->sc) != BBJD_SUCCESS) {
        delete o;
        return nullptr;
    }
    return o;
}

// Host callbacks (the reference's operator interface, include/bbjd.h:101-109):
// each application copies the operand to pinned host memory, calls back, and
// copies the result to the device.
struct CallbackOps : Operators {
    const bbjd_params *P;
    Scratch *S;
    cudaStream_t st;
    int *failed;
    zc *hx = nullptr, *hy = nullptr;
    int64_t n;
    CallbackOps(const bbjd_params *p, Scratch *s, cudaStream_t stream, int *f)
        : P(p), S(s), st(stream), failed(f), n(p->n) {}
    ~CallbackOps() override {
        cudaFreeHost(hx);
        cudaFreeHost(hy);
    }
    bbjd_status alloc() {
        BBJD_CUDA_TRY(cudaMallocHost(&hx, sizeof(zc) * n));
        BBJD_CUDA_TRY(cudaMallocHost(&hy, sizeof(zc) * n));
        return BBJD_SUCCESS;
    }
    bbjd_status call(bbjd_matvec_fn fn, const cplx *x, cplx *y, bool copy_in) {
        if (copy_in) {
            BBJD_CUDA_TRY(cudaMemcpyAsync(hx, x, sizeof(zc) * n, cudaMemcpyDeviceToHost, st));
            BBJD_CUDA_TRY(cudaStreamSynchronize(st));
        }
        if (*failed || fn(n, hx, hy, P->op_data)) {
            *failed = 1;
            return BBJD_ERR_CALLBACK;
        }
        BBJD_CUDA_TRY(cudaMemcpyAsync(y, hy, sizeof(zc) * n, cudaMemcpyHostToDevice, st));
        BBJD_CUDA_TRY(cudaStreamSynchronize(st));  // hy is reused by the next call
        return BBJD_SUCCESS;
    }
    bbjd_status apply(const cplx *x, cplx *yA, cplx *yB, cplx ta, cplx tb, cplx *r,
                      double *rnorm_dev) override {
        bbjd_status s = call(P->matvec_A, x, yA, true);
        if (s) return s;
        s = call(P->matvec_B, x, yB, false);
        if (s) return s;
        if (!r) return BBJD_SUCCESS;
        return update(*S, 0, n, nullptr, nullptr, nullptr, mk(0, 0), mk(0, 0), tb, yA,
                      mk(-ta.x, -ta.y), yB, r, rnorm_dev, nullptr, nullptr, nullptr, nullptr, st);
    }
    bool has_precond() const override { return P->precond != nullptr; }
    bbjd_status precond(int nrhs, const cplx *r, cplx *x) override {
        for (int q = 0; q < nrhs; ++q) {
            bbjd_status s = call(P->precond, r + (int64_t)q * n, x + (int64_t)q * n, true);
            if (s) return s;
        }
        return BBJD_SUCCESS;
    }
    double apply_bytes(bool residual) const override { return 16.0 * n * (residual ? 5 : 3); }
    double precond_bytes(int nrhs) const override { return 32.0 * n * nrhs; }
};

Operators *make_callback_ops(const bbjd_params *p, Scratch *S, cudaStream_t st, int *cb_failed) {
    auto *o = new (std::nothrow) CallbackOps(p, S, st, cb_failed);
    if (o && o->alloc() != BBJD_SUCCESS) {
        delete o;
        return nullptr;
    }
    return o;
}

static bbjd_status alloc_result(const bbjd_params *p, bbjd_result *r) {
    r->nconv = 0;
    r->iters = 0;
    r->status = BBJD_SUCCESS;
    r->eigenvalues = (bbjd_zomplex *)calloc((size_t)p->nev, sizeof(bbjd_zomplex));
    r->eigenvectors = (bbjd_zomplex *)calloc((size_t)p->n * p->nev, sizeof(bbjd_zomplex));
    r->residuals = (double *)calloc((size_t)p->nev, sizeof(double));
    if (!r->eigenvalues || !r->eigenvectors || !r->residuals) {
        bbjd_result_free(r);
        return BBJD_ERR_ALLOC;
    }
    return BBJD_SUCCESS;
}

static bool params_ok(const bbjd_params *p, const bbjd_workspace *ws) {
    return p && ws && p->n >= 1 && p->nev >= 1 && p->nev <= p->n && ws->n == p->n &&
           ws->nev >= p->nev && p->tol > 0 && p->maxiter >= 0;
}

extern "C" int scipy_openblas_get_num_threads(void);
extern "C" void scipy_openblas_set_num_threads(int);

// The k x k projected solves (k <= a few hundred) run fastest on one BLAS
// thread: at these sizes the pool's fork/join costs more than it saves
// (ZHSEQR at k = 140: 11.7 ms on 1 thread, 13.4 ms on 8).  While a device
// solve runs, the LAPACK library the engine links is held at one thread;
// the caller's setting comes back when the last concurrent solve returns.
// Callback-mode solves leave it alone, since the caller's own host code
// runs inside them.
class BlasOneThread {
public:
    BlasOneThread() {
        std::lock_guard<std::mutex> g(mu());
        if (users()++ == 0) {
            saved() = scipy_openblas_get_num_threads();
            scipy_openblas_set_num_threads(1);
        }
    }
    ~BlasOneThread() {
        std::lock_guard<std::mutex> g(mu());
        if (--users() == 0) scipy_openblas_set_num_threads(saved());
    }
private:
    static std::mutex &mu() { static std::mutex m; return m; }
    static int &users() { static int u = 0; return u; }
    static int &saved() { static int v = 1; return v; }
};

// Runs one engine solve; fills the extension's instrumentation.
static bbjd_status run_engine(const bbjd_params *p, bbjd_workspace *ws, bbjd_result *r,
                              bbjd_device_ext *ext, Operators *ops, Engine &E, cudaStream_t st,
                              int *cb_failed) {
    auto t0 = std::chrono::steady_clock::now();
    const long long l0 = g_launches.load();
    bbjd_status s = E.init(p, ws, r, ext, ops, st);
    if (s == BBJD_SUCCESS) s = E.run();
    if (p->verbose >= 1 && E.proj_mode == BBJD_PROJ_SCHUR)
        fprintf(stderr, "  projected solve %.3f s: form H %.3f, Hessenberg %.3f, eigenvalues %.3f, "
                "target vector %.3f, restart Schur form + reorder %.3f (FP32 estimates: %lld "
                "refinement LUs, %lld FP64 fallbacks); on the driving thread %.3f s; guesses %lld held, "
                "%lld rejected\n", E.qz_seconds, E.qz_split[0],
                E.qz_split[1], E.qz_split[2], E.qz_split[3], E.qz_split[4], E.rq_lus, E.rq_fallbacks,
                E.qz_exposed, E.spec_hits, E.spec_misses);
    if (s != BBJD_ERR_CUDA && !(cb_failed && *cb_failed)) {
        const bbjd_status f = E.finish_eigenvectors();
        if (f != BBJD_SUCCESS) s = f;
    }
    if (s == BBJD_ERR_CUDA || (cb_failed && *cb_failed)) {
        if (cb_failed && *cb_failed) s = BBJD_ERR_CALLBACK;
        r->status = s;
    }
    if (E.st) cudaStreamSynchronize(E.st);
    if (ext) {
        ext->seconds_total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        ext->seconds_qz = E.qz_seconds;
        ext->bytes_device = E.bytes_dev;
        ext->kernel_launches = g_launches.load() - l0;
        ext->dgks_passes = E.dgks;
        ext->restarts = E.restarts;
        ext->duplicates = E.duplicates;
        ext->ritz_refinements = E.rq_lus;
        ext->ritz_fallbacks = E.rq_fallbacks;
        ext->seconds_qz_exposed = E.qz_exposed;
        ext->guess_hits = E.spec_hits;
        ext->guess_misses = E.spec_misses;
        double dev = 0.0;
        E.T.flush();
        for (int c = 0; c < KC_N && c < 8; ++c) {
            ext->kernel_ms[c] = E.T.ms[c];
            ext->kernel_bytes[c] = E.T.bytes[c];
            ext->kernel_calls[c] = E.T.calls[c];
            dev += E.T.ms[c];
        }
        ext->seconds_device = dev * 1e-3;
        ext->seconds_restart = E.T.ms[KC_RESTART] * 1e-3;
    }
    E.release();
    if (s != BBJD_SUCCESS && s != BBJD_MAX_ITER && r->status >= 0) r->status = s;
    return r->status;
}

}  // namespace bbjd

using namespace bbjd;

extern "C" {

void bbjd_params_init(bbjd_params *p) {                // reference jd_core.c:73-84
    memset(p, 0, sizeof(*p));
    p->nev = 6;
    p->sigma = 0.0;
    p->target = BBJD_TARGET_NEAREST;
    p->tol = 1e-10;
    p->maxiter = 200;
    p->inner_maxiter = 0;
    p->inner_tol = 1e-2;
    p->v0 = nullptr;
}

void bbjd_device_ext_init(bbjd_device_ext *e) {
    memset(e, 0, sizeof(*e));
    e->precision = BBJD_FP64;
}

bbjd_workspace *bbjd_workspace_alloc(const bbjd_params *p) {   // reference jd_core.c:87-161
    if (!p || p->n < 1 || p->nev < 1) return nullptr;
    const bbjd_int n = p->n, nev = p->nev;
    bbjd_int maxsub_auto = 3 * nev + 10;
    if (maxsub_auto < 40) maxsub_auto = 40;
    const bbjd_int maxsub = p->maxsub > 0 ? p->maxsub : (maxsub_auto < n ? maxsub_auto : n);
    const bbjd_int ims = p->inner_maxiter > 0 ? p->inner_maxiter : 1;
    auto *ws = (bbjd_workspace *)calloc(1, sizeof(bbjd_workspace));
    if (!ws) return nullptr;
    ws->n = n;
    ws->maxsub = maxsub;
    ws->nev = nev;
    ws->inner_maxiter = ims;
    const size_t ns = (size_t)n * maxsub, ss = (size_t)maxsub * maxsub;
    bool ok = true;
    auto dalloc = [&](bbjd_zomplex **ptr, size_t count) {
        if (!ok) return;
        if (cudaMalloc((void **)ptr, sizeof(bbjd_zomplex) * (count ? count : 1)) != cudaSuccess) {
            *ptr = nullptr;
            ok = false;
        }
    };
    dalloc(&ws->V, ns);
    dalloc(&ws->W, ns);
    dalloc(&ws->AV, ns);
    dalloc(&ws->BV, ns);
    // the restart compresses V, AV and BV in place: no n x maxsub swap buffer
    ws->swap_nm = nullptr;
    dalloc(&ws->gmres_V, (size_t)n * (ims + 1));
    dalloc(&ws->tmp1, n);
    dalloc(&ws->tmp2, n);
    dalloc(&ws->tmp3, n);
    dalloc(&ws->tmp4, n);
    dalloc(&ws->Q_right, (size_t)n * (nev + 1));
    dalloc(&ws->Q_left, (size_t)n * (nev + 1));
    auto halloc = [&](bbjd_zomplex **ptr, size_t count) {
        *ptr = (bbjd_zomplex *)calloc(count ? count : 1, sizeof(bbjd_zomplex));
        if (!*ptr) ok = false;
    };
    halloc(&ws->MA, ss);
    halloc(&ws->MB, ss);
    halloc(&ws->SA, ss);
    halloc(&ws->SB, ss);
    halloc(&ws->ZA, ss);
    halloc(&ws->ZB, ss);
    halloc(&ws->gmres_H, (size_t)(ims + 1) * ims);
    halloc(&ws->gmres_cs, ims);
    halloc(&ws->gmres_sn, ims);
    halloc(&ws->gmres_g, ims + 1);
    halloc(&ws->h_work, (size_t)(2 * maxsub + nev + 4));
    if (!ok) {
        bbjd_workspace_free(ws);
        return nullptr;
    }
    return ws;
}

void bbjd_workspace_free(bbjd_workspace *ws) {
    if (!ws) return;
    cudaFree(ws->V); cudaFree(ws->W); cudaFree(ws->AV); cudaFree(ws->BV);
    cudaFree(ws->swap_nm); cudaFree(ws->gmres_V);
    cudaFree(ws->tmp1); cudaFree(ws->tmp2); cudaFree(ws->tmp3); cudaFree(ws->tmp4);
    cudaFree(ws->Q_right); cudaFree(ws->Q_left);
    free(ws->MA); free(ws->MB); free(ws->SA); free(ws->SB); free(ws->ZA); free(ws->ZB);
    free(ws->gmres_H); free(ws->gmres_cs); free(ws->gmres_sn); free(ws->gmres_g);
    free(ws->h_work);
    free(ws);
}

void bbjd_result_free(bbjd_result *r) {                 // reference jd_core.c:178-183
    if (!r) return;
    free(r->eigenvalues);
    free(r->eigenvectors);
    free(r->residuals);
    r->eigenvalues = nullptr;
    r->eigenvectors = nullptr;
    r->residuals = nullptr;
}

bbjd_status bbjd_solve(const bbjd_params *params, bbjd_workspace *ws, bbjd_result *result) {
    if (!result) return BBJD_ERR_INVALID;
    memset(result, 0, sizeof(*result));
    if (!params_ok(params, ws) || !params->matvec_A || !params->matvec_B)
        return result->status = BBJD_ERR_INVALID;
    bbjd_status s = alloc_result(params, result);
    if (s) return result->status = s;
    int failed = 0;
    Engine E;
    // the callback operators need the engine's scratch for the residual: the
    // engine initialises it, the operators borrow it through E.S.
    Operators *ops = make_callback_ops(params, &E.S, nullptr, &failed);
    if (!ops) return result->status = BBJD_ERR_ALLOC;
    // the callback operators must run on the engine's stream
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        delete ops;
        return result->status = BBJD_ERR_CUDA;
    }
    static_cast<CallbackOps *>(ops)->st = st;
    s = run_engine(params, ws, result, nullptr, ops, E, st, &failed);
    delete ops;
    cudaStreamDestroy(st);
    return s;
}

bbjd_status bbjd_solve_device(const bbjd_params *params, bbjd_device_ext *ext,
                              const bbjd_bbt_matrix *m, const bbjd_precond *pc,
                              bbjd_workspace *ws, bbjd_result *result) {
    if (!result) return BBJD_ERR_INVALID;
    memset(result, 0, sizeof(*result));
    if (!params_ok(params, ws) || !m || m->n != params->n) return result->status = BBJD_ERR_INVALID;
    if (pc && pc->n != m->n) return result->status = BBJD_ERR_INVALID;
    if (ext && ext->precision != BBJD_FP64 && ext->precision != BBJD_MIXED)
        return result->status = BBJD_ERR_INVALID;
    bbjd_status s = alloc_result(params, result);
    if (s) return result->status = s;
    cudaStream_t st = ext ? (cudaStream_t)ext->stream : nullptr;
    bool own = false;
    if (!st) {
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
            return result->status = BBJD_ERR_CUDA;
        own = true;
    }
    Engine E;
    Operators *ops = make_device_ops(m, pc, &E.S, st);
    if (!ops) return result->status = BBJD_ERR_ALLOC;
    {
        BlasOneThread one;
        s = run_engine(params, ws, result, ext, ops, E, st, nullptr);
    }
    delete ops;
    if (own) cudaStreamDestroy(st);
    return s;
}

bbjd_status bbjd_solve_batch(int count, const bbjd_params *params, bbjd_device_ext *exts,
                             const bbjd_bbt_matrix *const *mats, const bbjd_precond *const *pcs,
                             bbjd_workspace *const *wss, bbjd_result *results, int threads) {
    if (count < 0 || (count > 0 && (!params || !mats || !pcs || !wss || !results)) || threads < 1)
        return BBJD_ERR_INVALID;
    for (int i = 0; i < count; ++i) {
        if (!params[i].v0 || !mats[i] || !wss[i]) return BBJD_ERR_INVALID;
        for (int j = 0; j < i; ++j)
            if ((pcs[i] && pcs[j] == pcs[i]) || wss[j] == wss[i]) return BBJD_ERR_INVALID;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return BBJD_ERR_CUDA;
    // Largest solves first (cost ~ n x maxiter x maxsub, known up front):
    // the threads then finish close together instead of one long solve
    // starting last.  Results stay at their input positions.
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    auto cost = [&](int i) {
        return (double)params[i].n * (double)params[i].maxiter * (double)std::max<bbjd_int>(params[i].maxsub, 1);
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::atomic<int> next{0};
    std::vector<bbjd_status> st(count, BBJD_SUCCESS);
    const int nt = std::min(threads, std::max(count, 1));
    auto worker = [&]() {
        cudaSetDevice(dev);
        g_concurrent_solve = true;
        for (;;) {
            const int q = next.fetch_add(1);
            if (q >= count) break;
            const int i = order[q];
            bbjd_device_ext local;
            bbjd_device_ext_init(&local);
            bbjd_device_ext *e = exts ? &exts[i] : &local;
            st[i] = bbjd_solve_device(&params[i], e, mats[i], pcs[i], wss[i], &results[i]);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t) pool.emplace_back(worker);
    for (auto &th : pool) th.join();
    bbjd_status out = BBJD_SUCCESS;
    for (int i = 0; i < count; ++i) {
        if (st[i] < 0) return st[i];
        if (st[i] == BBJD_MAX_ITER) out = BBJD_MAX_ITER;
    }
    return out;
}

// Reference jd_core.c:244-266 on host arrays (staged through the device).
double bbjd_mgs_orthogonalize(bbjd_int n, bbjd_int k, const bbjd_zomplex *Q, bbjd_zomplex *v) {
    double nrm = -1.0;
    cplx *dQ = nullptr, *dv = nullptr;
    if (cudaMalloc(&dQ, sizeof(cplx) * (size_t)n * (k > 0 ? k : 1)) != cudaSuccess) return -1.0;
    if (cudaMalloc(&dv, sizeof(cplx) * (size_t)n) != cudaSuccess) { cudaFree(dQ); return -1.0; }
    if (k > 0) cudaMemcpy(dQ, Q, sizeof(cplx) * (size_t)n * k, cudaMemcpyHostToDevice);
    cudaMemcpy(dv, v, sizeof(cplx) * (size_t)n, cudaMemcpyHostToDevice);
    int second = 0;
    if (bbjd_dev_orthogonalize(n, k, reinterpret_cast<bbjd_zomplex *>(dQ), n,
                               reinterpret_cast<bbjd_zomplex *>(dv), &nrm, &second, nullptr) == BBJD_SUCCESS)
        cudaMemcpy(v, dv, sizeof(cplx) * (size_t)n, cudaMemcpyDeviceToHost);
    else
        nrm = -1.0;
    cudaFree(dQ);
    cudaFree(dv);
    return nrm;
}

bbjd_status bbjd_dev_orthogonalize(bbjd_int n, bbjd_int k, const bbjd_zomplex *Q, bbjd_int ldq,
                                   bbjd_zomplex *v, double *norm_out, int *second_pass_out,
                                   void *stream) {
    if (n < 1 || k < 0 || (k > 0 && (!Q || ldq < n)) || !v) return BBJD_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    Scratch S;
    bbjd_status s = S.init(n, (int)std::max<bbjd_int>(k, 1), 2);
    if (s) { S.release(); return s; }
    const cplx *dQ = reinterpret_cast<const cplx *>(Q);
    cplx *dv = reinterpret_cast<cplx *>(v);
    if (k == 0) {
        s = update(S, 0, n, nullptr, nullptr, nullptr, mk(0, 0), mk(0, 0), mk(1, 0), dv, mk(0, 0), nullptr,
                   dv, S.scal, nullptr, nullptr, nullptr, nullptr, st);
    } else {
        s = tsdot(S, 1, 1, (int)k, ldq, dQ, nullptr, dv, nullptr, S.red, nullptr, st);
        if (!s) s = cgs_tail(S, (int)k, ldq, dQ, S.red, nullptr, mk(1, 0), mk(0, 0), mk(1, 0), dv, mk(0, 0),
                             nullptr, dv, S.scal, S.red + k, nullptr, S.flags, S.red + S.maxX, st);
    }
    double nrm = 0.0;
    int flag = 0, tmo = 0;
    if (!s && cudaMemcpyAsync(&nrm, S.scal, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess) s = BBJD_ERR_CUDA;
    if (!s && k > 0 && cudaMemcpyAsync(&flag, S.flags, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) s = BBJD_ERR_CUDA;
    if (!s && cudaMemcpyAsync(&tmo, S.flags + SCRATCH_FLAG_TMO, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        s = BBJD_ERR_CUDA;
    if (!s && cudaStreamSynchronize(st) != cudaSuccess) s = BBJD_ERR_CUDA;
    if (!s && tmo) s = BBJD_ERR_DEVICE_TIMEOUT;
    S.release();
    if (norm_out) *norm_out = nrm;
    if (second_pass_out) *second_pass_out = flag;
    return s;
}

static bbjd_status dev_restart_gemm(bbjd_int n, bbjd_int k, bbjd_int keep, const bbjd_zomplex *X,
                                    bbjd_int ldx, const bbjd_zomplex *Z_host, bbjd_int ldz,
                                    bbjd_zomplex *out, void *stream, bool stalled) {
    if (n < 1 || k < 1 || keep < 1 || !X || !Z_host || !out || ldz < k || ldx < n) return BBJD_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    cplx *dZ = nullptr;
    std::vector<cplx> zh((size_t)k * keep);
    for (bbjd_int c = 0; c < keep; ++c)
        for (bbjd_int i = 0; i < k; ++i) zh[c * k + i] = mk(Z_host[i + c * ldz].real(), Z_host[i + c * ldz].imag());
    int *derr = nullptr;
    BBJD_CUDA_TRY(cudaMalloc(&dZ, sizeof(cplx) * zh.size()));
    BBJD_CUDA_TRY(cudaMalloc(&derr, sizeof(int)));
    BBJD_CUDA_TRY(cudaMemset(derr, 0, sizeof(int)));
    BBJD_CUDA_TRY(cudaMemcpy(dZ, zh.data(), sizeof(cplx) * zh.size(), cudaMemcpyHostToDevice));
    // the solver's form: TMA-staged where keep <= 128, with its timeout flag
    bbjd_status s = stalled ? restart_gemm_stalled(n, (int)k, (int)keep, reinterpret_cast<const cplx *>(X),
                                                   ldx, dZ, (int)k, reinterpret_cast<cplx *>(out), st, derr)
                            : restart_gemm(n, (int)k, (int)keep, reinterpret_cast<const cplx *>(X), ldx, dZ,
                                           (int)k, reinterpret_cast<cplx *>(out), st, derr);
    int herr = 0;
    if (!s && (cudaStreamSynchronize(st) != cudaSuccess ||
               cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess))
        s = BBJD_ERR_CUDA;
    if (!s && herr) s = BBJD_ERR_DEVICE_TIMEOUT;
    cudaFree(dZ);
    cudaFree(derr);
    return s;
}

bbjd_status bbjd_dev_restart_gemm(bbjd_int n, bbjd_int k, bbjd_int keep, const bbjd_zomplex *X,
                                  bbjd_int ldx, const bbjd_zomplex *Z_host, bbjd_int ldz,
                                  bbjd_zomplex *out, void *stream) {
    return dev_restart_gemm(n, k, keep, X, ldx, Z_host, ldz, out, stream, false);
}

bbjd_status bbjd_dev_restart_gemm_stalled(bbjd_int n, bbjd_int k, bbjd_int keep, const bbjd_zomplex *X,
                                          bbjd_int ldx, const bbjd_zomplex *Z_host, bbjd_int ldz,
                                          bbjd_zomplex *out, void *stream) {
    if (keep > 80) return BBJD_ERR_INVALID;
    return dev_restart_gemm(n, k, keep, X, ldx, Z_host, ldz, out, stream, true);
}

bbjd_status bbjd_dev_gram(bbjd_int n, bbjd_int keep, const bbjd_zomplex *X, const bbjd_zomplex *Y,
                          bbjd_int ldx, bbjd_zomplex *C_host, bbjd_int ldc, void *stream) {
    if (n < 1 || keep < 1 || !X || !Y || !C_host || ldc < keep || ldx < n) return BBJD_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    Scratch S;
    bbjd_status s = S.init(n, 1, 1);
    const int Gg = (int)std::max<int64_t>(1, std::min<int64_t>(num_sms(), (n + 1023) / 1024));
    cplx *part = nullptr, *out = nullptr;
    if (!s && cudaMalloc(&part, sizeof(cplx) * (size_t)Gg * keep * keep) != cudaSuccess) s = BBJD_ERR_ALLOC;
    if (!s && cudaMalloc(&out, sizeof(cplx) * (size_t)keep * keep) != cudaSuccess) s = BBJD_ERR_ALLOC;
    if (!s) s = gram(S, (int)keep, reinterpret_cast<const cplx *>(X), reinterpret_cast<const cplx *>(Y), ldx,
                     part, Gg, out, st);
    std::vector<cplx> h((size_t)keep * keep);
    if (!s && cudaMemcpyAsync(h.data(), out, sizeof(cplx) * h.size(), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        s = BBJD_ERR_CUDA;
    if (!s && cudaStreamSynchronize(st) != cudaSuccess) s = BBJD_ERR_CUDA;
    if (!s)
        for (bbjd_int c = 0; c < keep; ++c)
            for (bbjd_int i = 0; i < keep; ++i) C_host[i + c * ldc] = bbjd_zomplex(h[c * keep + i].x, h[c * keep + i].y);
    cudaFree(part);
    cudaFree(out);
    S.release();
    return s;
}

// Reference jd_core.c:568-727 on host arrays: the projectors, r and z are
// host memory; the Arnoldi basis lives in ws->gmres_V on the device.
int bbjd_correction_gmres(bbjd_int n, const bbjd_zomplex *q, const bbjd_zomplex *p,
                          bbjd_zomplex theta_a, bbjd_zomplex theta_b, const bbjd_zomplex *r,
                          bbjd_zomplex *z, bbjd_matvec_fn matvec_A, bbjd_matvec_fn matvec_B,
                          bbjd_precond_fn precond, void *op_data, bbjd_int maxiter, double tol,
                          bbjd_workspace *ws) {
    if (!ws || ws->n != n || !q || !p || !r || !z || !matvec_A || !matvec_B || maxiter < 1 ||
        maxiter > ws->inner_maxiter)
        return -1;
    bbjd_params prm;
    bbjd_params_init(&prm);
    prm.n = n;
    prm.nev = ws->nev;
    prm.maxsub = ws->maxsub;
    prm.tol = 1e-10;
    prm.inner_maxiter = maxiter;
    prm.inner_tol = tol;
    prm.matvec_A = matvec_A;
    prm.matvec_B = matvec_B;
    prm.precond = precond;
    prm.op_data = op_data;
    const int64_t ndefl = ws->nlock + 1;
    bbjd_result res;
    memset(&res, 0, sizeof(res));
    int failed = 0;
    Engine E;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return -1;
    Operators *ops = make_callback_ops(&prm, &E.S, st, &failed);
    int rc = -1;
    if (ops && E.init(&prm, ws, &res, nullptr, ops, st) == BBJD_SUCCESS) {
        const size_t nv = sizeof(cplx) * (size_t)n;
        bool ok = cudaMemcpy(ws->Q_right, q, nv * ndefl, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(ws->Q_left, p, nv * ndefl, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(E.ru, r, nv, cudaMemcpyHostToDevice) == cudaSuccess;
        if (ok && E.gmres((int)ndefl, zc(theta_a), zc(theta_b), E.ru, E.g3) == BBJD_SUCCESS && !failed) {
            cudaStreamSynchronize(st);
            if (cudaMemcpy(z, E.g3, nv, cudaMemcpyDeviceToHost) == cudaSuccess) rc = 0;
        }
    }
    E.release();
    delete ops;
    cudaStreamDestroy(st);
    return rc;
}

const char *bbjd_gpu_version(void) {
    return "bbjd_gpu 0.1 (sm_100a, FP64 engine, host LAPACK QZ)";
}

}  // extern "C"
