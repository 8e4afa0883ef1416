// run.cu -- many bi-conjugate Lanczos steps over several systems (ensembles) without returning to
// the host: the loop of Lanczos.run_FT (Modules/DynamicalLanczos.py:5843-6374, n_rep_orth = 0)
// for every chain of every system, advanced in lockstep.
//
// One step of one system (nc chains, len = n + n(n+1)):
//   [L q_c ; L^T p_c]  = apply_full_L over the 2 nc vectors [q; p]   (one batched apply)
//   q', p', a, b, c    = the bi-conjugate recurrence                   (lanczos_step_device)
//   history, (a, b, c) record, q_prev <- q, q <- q'                   (run_advance_kernel + 2 copies)
// Systems run on their own streams, forked from and joined back into the caller's stream, so the
// small systems' kernels fill the SMs the large system's contraction leaves idle.  With use_graph
// the first two steps run eagerly (they tune the contraction tiles, allocate the workspaces and fix
// the chunking plans) and all remaining steps of all systems are captured into one CUDA graph that
// is launched once: the rest of the run is a single launch from the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "apply.cuh"
#include "common.cuh"
#include "ensemble.cuh"

namespace tdscha {
namespace {

constexpr int RUN_MAX_CHAINS = 32;     // 2 nc <= 64 vectors per batched apply
constexpr int RUN_MAX_SYSTEMS = 16;

constexpr double RUN_BREAKDOWN = 1e-12;   // |b| or |c| below it ends a chain (run_FT's __EPSILON__)

// sc (nc, 6) = [c_{k-1}, b_{k-1}, s_norm_k, s_norm_{k-1}, c_{k-2}, k]; sc_out (nc, 4) =
// [a_k, b_k, c_k, s_norm_{k+1}].  For every chain still running: records sc_out at row *counter of
// coef, then either marks the chain done (breakdown: |b| or |c| < 1e-12, the step's a_k is its last
// coefficient, as in run_FT) or advances its history.  Chains already done record nothing.
__global__ void run_advance_kernel(int nc, double *__restrict__ sc, const double *__restrict__ sc_out,
                                   double *__restrict__ coef, int *__restrict__ done, int *__restrict__ counter, int n_steps) {
    const int c = threadIdx.x;
    const int k = *counter;
    if (c < nc && !done[c]) {
        const double a = sc_out[4 * c], b = sc_out[4 * c + 1], cc = sc_out[4 * c + 2], s = sc_out[4 * c + 3];
        if (k < n_steps) {
            double *row = coef + ((long long)k * nc + c) * 4;
            row[0] = a;
            row[1] = b;
            row[2] = cc;
            row[3] = s;
        }
        if (!(fabs(b) >= RUN_BREAKDOWN && fabs(cc) >= RUN_BREAKDOWN)) {   // NaN counts as a breakdown
            done[c] = 1;
        } else {
            double *h = sc + 6 * c;
            const double step = h[5], c_prev = h[0], s_cur = h[2];
            h[4] = step >= 1.0 ? c_prev : 1.0;
            h[3] = s_cur;
            h[0] = cc;
            h[1] = b;
            h[2] = s;
            h[5] = step + 1.0;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter = k + 1;
}

// [q; p] -> [q_prev; p_prev] and [q'; p'] -> [q; p] for the chains still running (a chain that
// broke down keeps its last vectors).  qp: (4, nc, len) = q, p, q_prev, p_prev; next: (2, nc, len).
__global__ void run_rotate_kernel(int nc, long long len, double *__restrict__ qp, const double *__restrict__ next,
                                  const int *__restrict__ done) {
    const long long half = 2LL * nc * len;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < half;
         idx += (long long)gridDim.x * blockDim.x) {
        const int c = (int)((idx / len) % nc);
        if (done[c]) continue;
        const double cur = qp[idx];
        qp[half + idx] = cur;
        qp[idx] = next[idx];
    }
}

struct SysWork {
    double *out = nullptr;      // (2 nc, len) apply output
    double *next = nullptr;     // (2 nc, len) q', p'
    double *sc_out = nullptr;   // (nc, 4)
    double *apply_work = nullptr;
    size_t apply_bytes = 0;
    double *lz = nullptr;
    size_t lz_bytes = 0;
    int *tr = nullptr;          // (2 nc) transpose flags: nc zeros, nc ones
    int *counter = nullptr;
    int *done = nullptr;        // (nc) chain ended by a breakdown
    cudaStream_t stream = nullptr;
    cudaEvent_t joined = nullptr;
};

struct RunState {
    std::vector<SysWork> w;
    cudaEvent_t fork = nullptr;
    ~RunState() {
        for (SysWork &s : w)
            if (s.stream) cudaStreamSynchronize(s.stream);   // nothing in flight uses the buffers below
        for (SysWork &s : w) {
            cudaFree(s.out);
            cudaFree(s.next);
            cudaFree(s.sc_out);
            cudaFree(s.apply_work);
            cudaFree(s.lz);
            cudaFree(s.tr);
            cudaFree(s.counter);
            cudaFree(s.done);
            if (s.joined) cudaEventDestroy(s.joined);
        }
        if (fork) cudaEventDestroy(fork);
    }
};

// The systems' streams, created once per (device, system slot) and kept for the process (the
// contraction keys its tile-start counters by stream).
std::mutex g_run_mutex;
cudaStream_t g_run_streams[64][RUN_MAX_SYSTEMS + 1] = {};   // + the run's own origin stream

int run_stream(int dev, int slot, cudaStream_t *out) {
    TD_CHECK(dev >= 0 && dev < 64, TDSCHA_EINVAL, "device index %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_run_mutex);
    if (!g_run_streams[dev][slot]) TD_CUDA(cudaStreamCreateWithFlags(&g_run_streams[dev][slot], cudaStreamNonBlocking));
    *out = g_run_streams[dev][slot];
    return 0;
}

long long vec_len(const tdscha_ensemble *e) { return (long long)e->n + (long long)e->n * (e->n + 1); }

int enqueue_system_step(const tdscha_run_system &sy, SysWork &w, int n_steps) {
    const int nc = sy.n_chains, nb = 2 * nc;
    const long long len = vec_len(sy.ens);
    cudaStream_t st = w.stream;
    double *q = sy.qp, *p = sy.qp + (size_t)nc * len, *qprev = sy.qp + 2 * (size_t)nc * len,
           *pprev = sy.qp + 3 * (size_t)nc * len;
    TD_TRY(apply_full_L_device_flags(sy.ens, nb, sy.qp, w.tr, &sy.opts, sy.precision, w.out, st, w.apply_work, w.apply_bytes));
    TD_TRY(lanczos_step_device(nc, len, w.out, w.out + (size_t)nc * len, q, p, qprev, pprev, sy.sc, nullptr, w.next,
                               w.next + (size_t)nc * len, w.sc_out, st, w.lz, w.lz_bytes));
    run_advance_kernel<<<1, 32, 0, st>>>(nc, sy.sc, w.sc_out, sy.coef, w.done, w.counter, n_steps);
    const long long elems = (long long)nb * len;
    run_rotate_kernel<<<(unsigned)std::min<long long>((elems + 255) / 256, 148LL * 16), 256, 0, st>>>(nc, len, sy.qp, w.next,
                                                                                                       w.done);
    TD_CUDA(cudaGetLastError());
    return 0;
}

// One step of every system: fork from `st` to the systems' streams, join back.
int enqueue_step(int ns, const tdscha_run_system *sys, RunState &rs, int n_steps, cudaStream_t st) {
    TD_CUDA(cudaEventRecord(rs.fork, st));
    for (int i = 0; i < ns; ++i) {
        TD_CUDA(cudaStreamWaitEvent(rs.w[i].stream, rs.fork, 0));
        TD_TRY(enqueue_system_step(sys[i], rs.w[i], n_steps));
        TD_CUDA(cudaEventRecord(rs.w[i].joined, rs.w[i].stream));
    }
    for (int i = 0; i < ns; ++i) TD_CUDA(cudaStreamWaitEvent(st, rs.w[i].joined, 0));
    return 0;
}

int check_err_words(int ns, const tdscha_run_system *sys, cudaStream_t st) {
    for (int i = 0; i < ns; ++i) {
        unsigned h = 0;
        TD_CUDA(cudaMemcpyAsync(&h, sys[i].ens->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        TD_CUDA(cudaStreamSynchronize(st));
        if (h) {
            cudaMemsetAsync(sys[i].ens->d_err, 0, sizeof(unsigned), st);
            set_error("system %d: a tensor-core kernel hit its bounded-wait limit and aborted (error word 0x%x)", i, h);
            return TDSCHA_ETIMEOUT;
        }
    }
    return 0;
}

}  // namespace

int lanczos_run_device(int ns, const tdscha_run_system *sys, int n_steps, int use_graph, cudaStream_t caller) {
    TD_CHECK(ns >= 1 && ns <= RUN_MAX_SYSTEMS, TDSCHA_EINVAL, "1..%d systems per run (got %d)", RUN_MAX_SYSTEMS, ns);
    TD_CHECK(sys != nullptr && n_steps >= 0, TDSCHA_EINVAL, "bad run arguments");
    for (int i = 0; i < ns; ++i) {
        const tdscha_run_system &s = sys[i];
        TD_CHECK(s.ens && s.qp && s.sc && s.coef, TDSCHA_EINVAL, "system %d: NULL argument", i);
        TD_CHECK(s.n_chains >= 1 && s.n_chains <= RUN_MAX_CHAINS, TDSCHA_EINVAL, "system %d: 1..%d chains (got %d)", i,
                 RUN_MAX_CHAINS, s.n_chains);
        TD_CHECK(s.precision >= TDSCHA_PREC_FP64 && s.precision <= TDSCHA_PREC_BF16, TDSCHA_EINVAL,
                 "system %d: unknown precision %d", i, s.precision);
        TD_CHECK(s.ens->device == sys[0].ens->device, TDSCHA_EINVAL, "all systems of a run must be on one device");
        for (int j = 0; j < i; ++j) TD_CHECK(sys[j].ens != s.ens, TDSCHA_EINVAL, "systems %d and %d share an ensemble", j, i);
    }
    if (n_steps == 0) return 0;
    TD_CUDA(cudaSetDevice(sys[0].ens->device));
    RunState rs;
    rs.w.resize(ns);
    TD_CUDA(cudaEventCreateWithFlags(&rs.fork, cudaEventDisableTiming));
    // the run's own origin stream (a capture cannot start on the legacy default stream), ordered
    // after the caller's stream
    cudaStream_t st = nullptr;
    TD_TRY(run_stream(sys[0].ens->device, RUN_MAX_SYSTEMS, &st));
    TD_CUDA(cudaEventRecord(rs.fork, caller));
    TD_CUDA(cudaStreamWaitEvent(st, rs.fork, 0));
    for (int i = 0; i < ns; ++i) {
        const tdscha_run_system &s = sys[i];
        SysWork &w = rs.w[i];
        const int nc = s.n_chains, nb = 2 * nc;
        const long long len = vec_len(s.ens);
        const size_t n = s.ens->n;
        TD_TRY(run_stream(s.ens->device, i, &w.stream));
        TD_CUDA(cudaEventCreateWithFlags(&w.joined, cudaEventDisableTiming));
        TD_CUDA(cudaMalloc(&w.out, (size_t)nb * len * sizeof(double)));
        TD_CUDA(cudaMalloc(&w.next, (size_t)nb * len * sizeof(double)));
        TD_CUDA(cudaMalloc(&w.sc_out, (size_t)nc * 4 * sizeof(double)));
        w.apply_bytes = (size_t)nb * (2 * n + 2 * n * n) * sizeof(double);
        TD_CUDA(cudaMalloc(&w.apply_work, w.apply_bytes));
        w.lz_bytes = lanczos_scratch_bytes(nc);
        TD_CUDA(cudaMalloc(&w.lz, w.lz_bytes));
        TD_CUDA(cudaMalloc(&w.tr, nb * sizeof(int)));
        TD_CUDA(cudaMalloc(&w.counter, sizeof(int)));
        TD_CUDA(cudaMalloc(&w.done, nc * sizeof(int)));
        TD_CUDA(cudaMemset(w.done, 0, nc * sizeof(int)));
        std::vector<int> tr(nb, 0);
        for (int c = nc; c < nb; ++c) tr[c] = 1;
        TD_CUDA(cudaMemcpy(w.tr, tr.data(), nb * sizeof(int), cudaMemcpyHostToDevice));
        TD_CUDA(cudaMemset(w.counter, 0, sizeof(int)));
    }
    // profiling events cannot be read back from graph replays: off for the run
    std::vector<bool> prof_on(ns);
    for (int i = 0; i < ns; ++i) {
        prof_on[i] = sys[i].ens->prof.enabled;
        sys[i].ens->prof.enabled = false;
    }
    struct Restore {
        const tdscha_run_system *sys;
        std::vector<bool> &on;
        ~Restore() {
            for (size_t i = 0; i < on.size(); ++i) sys[i].ens->prof.enabled = on[i];
        }
    } restore{sys, prof_on};

    const int eager = use_graph ? std::min(n_steps, 2) : n_steps;
    for (int k = 0; k < eager; ++k) TD_TRY(enqueue_step(ns, sys, rs, n_steps, st));
    if (eager < n_steps) {
        TD_TRY(check_err_words(ns, sys, st));   // also completes the eager steps
        // the remaining steps go into as few graphs as possible: `per` consecutive steps of all
        // systems are captured into one graph (TDSCHA_RUN_GRAPH_STEPS caps it; by default all
        // remaining steps, i.e. a single graph launch for the rest of the run), and a shorter graph
        // takes the remainder
        const int rem = n_steps - eager;
        const char *env = getenv("TDSCHA_RUN_GRAPH_STEPS");
        const int cap_steps = env && atoi(env) > 0 ? atoi(env) : rem;
        const int per = std::min(rem, cap_steps);
        auto build = [&](int steps, cudaGraphExec_t *exec) -> int {
            cudaGraph_t graph = nullptr;
            TD_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
            int rc = 0;
            for (int k = 0; k < steps && rc == 0; ++k) rc = enqueue_step(ns, sys, rs, n_steps, st);
            const cudaError_t ec = cudaStreamEndCapture(st, &graph);
            if (rc != 0) {
                if (graph) cudaGraphDestroy(graph);
                return rc;
            }
            TD_CHECK(ec == cudaSuccess && graph, TDSCHA_ECUDA, "graph capture of run steps failed: %s", cudaGetErrorString(ec));
            const cudaError_t ei = cudaGraphInstantiate(exec, graph, 0);
            cudaGraphDestroy(graph);
            TD_CHECK(ei == cudaSuccess, TDSCHA_ECUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(ei));
            return 0;
        };
        cudaGraphExec_t full = nullptr, tail = nullptr;
        TD_TRY(build(per, &full));
        if (rem % per) {
            const int rc = build(rem % per, &tail);
            if (rc != 0) {
                cudaGraphExecDestroy(full);
                return rc;
            }
        }
        cudaError_t el = cudaSuccess;
        for (int k = 0; k + per <= rem && el == cudaSuccess; k += per) el = cudaGraphLaunch(full, st);
        if (tail && el == cudaSuccess) el = cudaGraphLaunch(tail, st);
        const cudaError_t es = cudaStreamSynchronize(st);
        cudaGraphExecDestroy(full);
        if (tail) cudaGraphExecDestroy(tail);
        TD_CHECK(el == cudaSuccess && es == cudaSuccess, TDSCHA_ECUDA, "graph launch failed: %s",
                 cudaGetErrorString(el != cudaSuccess ? el : es));
    }
    TD_TRY(check_err_words(ns, sys, st));   // synchronises st: the run is complete
    return 0;
}

}  // namespace tdscha
