// The JDQZ engine: host driver state shared by the device-operator and the
// host-callback entry points.
#pragma once

#include <chrono>
#include <complex>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "bbt.cuh"

namespace bbjd {

typedef std::complex<double> zc;

// Operators of one solve: A and B products (with the optional fused
// residual r = tb A x - ta B x and its norm) and the preconditioner.
struct Operators {
    virtual ~Operators() {}
    // yA = A x, yB = B x; if r: r = tb yA - ta yB and *rnorm_dev = ||r||.
    virtual bbjd_status apply(const cplx *x, cplx *yA, cplx *yB, cplx ta, cplx tb, cplx *r,
                              double *rnorm_dev) = 0;
    virtual bool has_precond() const = 0;
    // x[:, q] = M^-1 r[:, q] for q < nrhs (stride n).
    virtual bbjd_status precond(int nrhs, const cplx *r, cplx *x) = 0;
    virtual double apply_bytes(bool residual) const = 0;
    virtual double precond_bytes(int nrhs) const = 0;
};

Operators *make_device_ops(const bbjd_bbt_matrix *m, const bbjd_precond *pc, Scratch *S,
                           cudaStream_t st);
Operators *make_callback_ops(const bbjd_params *p, Scratch *S, cudaStream_t st, int *cb_failed);

// Set on the host threads of bbjd_solve_batch: their projected solves take
// the OpenBLAS path (with a solve on every core, MKL's ZGEEV was measured
// slower than OpenBLAS on the B200 host; alone it is faster), whatever the
// thread count, so a batch returns the same bits with 1 or N threads.
extern thread_local bool g_concurrent_solve;

enum KClass { KC_SPMV = 0, KC_ORTH, KC_PENCIL, KC_RITZ, KC_PRECOND, KC_RESTART, KC_SMALL, KC_GMRES, KC_N };

// Device timing of kernel classes with CUDA events on the solve's stream.
struct Timer {
    bool on = false;
    cudaStream_t st = nullptr;
    struct Rec { int cls; cudaEvent_t a, b; double bytes; };
    std::vector<Rec> pending;
    std::vector<cudaEvent_t> pool;
    double ms[KC_N] = {0}, bytes[KC_N] = {0};
    long long calls[KC_N] = {0};
    int cur_cls = -1;
    cudaEvent_t cur_a = nullptr;
    double cur_bytes = 0;
    cudaEvent_t get();
    void begin(int cls, double b);
    void end();
    void flush();   // after a stream sync
    void release();
};

// One host thread beside the thread that drives the device: it computes the
// complex64 eigenvalue estimates of an outer iteration's projected matrix
// while the device works on the target guessed for that iteration.
struct HostWorker {
    std::thread th;
    std::mutex m;
    std::condition_variable cv;
    std::function<void()> job;
    bool busy = false, quit = false;
    void submit(std::function<void()> f);
    void wait();
    void stop();
    ~HostWorker() { stop(); }
};

struct Engine {
    const bbjd_params *P = nullptr;
    bbjd_workspace *ws = nullptr;
    bbjd_result *res = nullptr;
    bbjd_device_ext *ext = nullptr;
    Operators *ops = nullptr;
    Scratch S;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    Timer T;

    int64_t n = 0, maxsub = 0, nev = 0, minsub = 0;
    zc sigma, nu0, mu0;
    int target = 0;
    double tol = 0;

    // device buffers owned by the engine
    cplx *ru = nullptr;    // [r | u]  (2n)
    cplx *zs = nullptr;    // [z | s]  (2n)
    cplx *Au = nullptr, *Bu = nullptr;
    cplx *g1 = nullptr, *g2 = nullptr, *g3 = nullptr;  // GMRES / scratch vectors
    cplx *Zdev = nullptr;  // maxsub x maxsub restart coefficients
    cplx *xdev = nullptr;  // maxsub Ritz / combination coefficients
    cplx *gram_part = nullptr;
    int gram_G = 0;
    cplx *gram_out = nullptr;  // 2 x maxsub^2
    double *dscal = nullptr;   // device scalars
    int *dflag = nullptr;      // device flags
    bool mixed = false;        // BBJD_MIXED: complex64 shadow of V for the first CGS pass
    float2 *Vs = nullptr;      // n x maxsub complex64 copy of V (ld n)
    float2 *gV32 = nullptr;    // BBJD_MIXED with inner GMRES: complex64 Arnoldi basis,
                               // n x (inner_maxiter + 1) (ld n)
    int evec_layout = BBJD_EVEC_COLUMN_MAJOR;
    cplx *evd = nullptr;       // BBJD_EVEC_ROW_MAJOR: converged vectors, n x nev (ld n)
    cplx *pin = nullptr;       // pinned host staging for small results
    double *pin_d = nullptr;
    int *pin_i = nullptr;

    // host LAPACK workspace of the projected solve
    std::vector<zc> alpha, beta, zwork;
    std::vector<double> rwork;
    std::vector<int> bwork, sel, iwork;
    // harmonic standard-form projected solve: C = nu0 MA + mu0 MB,
    // H = C^-1 MB = Q T Q^H (ld = maxsub); omega = eig(H)
    int proj_mode = BBJD_PROJ_QZ;
    bool schur_step = false;          // the last projected solve used the Schur form
    bool ritz_ready = false;          // hx holds the target's coefficients already
    std::vector<zc> hC, hT, hx, tau, omega;
    // H of the last Schur-form projected solve (k = hH_k, ld maxsub; 0 = none)
    // and the iterations since it was last formed in full
    std::vector<zc> hH, hxs, hys;
    int hH_k = 0, hH_age = 0;
    // complex64 copy of H and LAPACK workspace for the FP32 eigenvalue
    // estimates (BBJD_RITZ_FP32); refinement LU count and FP64 fallbacks
    bool ritz32 = true;
    std::vector<std::complex<float>> hC32, w32, zwork32, tau32;
    std::vector<float> rwork32;
    long long rq_lus = 0, rq_fallbacks = 0;
    std::vector<int> ipiv;
    // Target guessed from the previous one (the canonical rule of
    // pick_target): when the previous iteration's target vector, extended
    // by a zero, is nearly an eigenvector of the new H, Rayleigh-quotient
    // iteration from it gives (spec_w, hx) before the k estimates exist.  spec_async: the estimates then run on `worker` while the device
    // works on the guess, and are checked before the iteration commits.
    bool spec_async = false;
    bool has_prev = false;            // prev_x: the last committed target's eigenvector of H
    std::vector<zc> prev_x;           // (k - 1 entries; its residual was prev_rel)
    double prev_rel = 0;
    bool spec_ok = false;             // this iteration has a guess (spec_w, hx)
    zc spec_w;
    bool est_pending = false;         // estimates running on the worker
    bool est_ok = false;              // estimates finished and finite
    double est_seconds = 0;           // worker seconds of the pending estimates
    HostWorker worker;
    long long spec_hits = 0, spec_misses = 0;
    double qz_exposed = 0;            // projected-solve seconds on the driving thread
    double qz_seconds = 0;
    // host seconds of the Schur-form projected solve: forming H, Hessenberg
    // reduction, eigenvalues (QR), target vector, restart Schur form + reorder
    double qz_split[5] = {0, 0, 0, 0, 0};
    long long dgks = 0, restarts = 0, duplicates = 0;
    double bytes_dev = 0;
    // locked eigenvalues and the window within which a Ritz value matches one
    struct Lock { zc value; double window; };
    std::vector<Lock> locks;
    int lock_rule = BBJD_LOCK_ROBUST;
    double lock_rel = 1e-6;
    bool is_locked(zc lam) const {
        for (const auto &l : locks)
            if (std::abs(lam - l.value) < l.window) return true;
        return false;
    }

    bbjd_status init(const bbjd_params *p, bbjd_workspace *w, bbjd_result *r, bbjd_device_ext *e,
                     Operators *o, cudaStream_t stream);
    void release();
    bbjd_status run();

    // building blocks
    bbjd_status orthogonalize(const cplx *Q, int64_t ldq, int k, cplx *v, double *norm_dev,
                              int cls);
    bbjd_status orthogonalize_mixed(int k, cplx *v, double *norm_dev);
    bbjd_status project_out(const cplx *Q, int k, cplx *v, int cls);
    bbjd_status deflation_append(int j, const cplx *u, const cplx *Au_, const cplx *Bu_);
    int rebuild_W_cholqr(int keep);
    bbjd_status gmres(int ndefl, zc ta, zc tb, const cplx *r, cplx *z);
    bbjd_status gmres_mixed(int ndefl, zc ta, zc tb, const cplx *r, cplx *z);
    int solve_projected(int k, int locked, int nkeep, int *target_pos);
    int solve_projected_schur(int k, int nkeep, bool reorder, int *target_pos);
    void hessenberg_eigvec(int k, zc w, zc *x);
    void dense_eigvec(int k, zc w, zc *x, const zc *x0 = nullptr);
    bool eigenvalues32(int k);
    int form_H(int k);
    int eig_fp64(int k, int nkeep, bool reorder, int *target_pos);
    int projected_begin(int k, int nkeep, bool reorder, int *target_pos);
    int projected_resolve(int k, int *target_pos, bool *changed);
    int pick_target(int k, int *target_pos, bool *guessed);
    bool rq_refine(int k, zc &w, zc *x, const zc *x0 = nullptr, int max_lu = 5);
    bool refine_target(int k, int *target_pos);
    void to_lambda(int i);
    void lambda_of(zc w, zc &a, zc &b) const;
    void select_and_scan(int k, int nkeep, int *target_pos);
    void ritz_coefficients(int k, int p, zc ta, zc tb, cplx *x);
    bbjd_status sync();
    bbjd_status finish_eigenvectors();
    void second_pass_bytes(int cls, int k);
};

}  // namespace bbjd
