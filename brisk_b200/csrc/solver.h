// Host-side solver of the B200 SDP Newton step: the problem as given, the options, the result.
#pragma once
#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace bsolve {

// An allocator whose resize() leaves new elements uninitialised: the big arrays are written in
// full right after they are sized (in parallel), so a serial zero fill first would be wasted.
template <typename T>
struct NoInitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <typename U>
    NoInitAlloc(const NoInitAlloc<U> &) noexcept {}
    template <typename U>
    void construct(U *p) noexcept {
        ::new (static_cast<void *>(p)) U;
    }
    template <typename U, typename... Args>
    void construct(U *p, Args &&...args) {
        ::new (static_cast<void *>(p)) U(std::forward<Args>(args)...);
    }
};

// The numbers of an SDPA sparse problem (brisk.h:128-140), already checked and with zero
// values dropped.  mat 0 = F0 = -C; 1..m = A_i; i, j are 1-based within the block.
struct InputData {
    int m = 0, nblk = 0;
    std::vector<int> bs;
    std::vector<double> c;
    std::vector<int, NoInitAlloc<int>> mat, blk, i, j;
    std::vector<double, NoInitAlloc<double>> v;
};

// The same numbers seen in place (the caller's arrays; nothing copied; zero values are skipped
// as make_input does).
struct InputView {
    int m = 0, nblk = 0;
    const int *bs = nullptr;
    const double *c = nullptr;
    long long nnz = 0;
    const int *mat = nullptr, *blk = nullptr, *i = nullptr, *j = nullptr;
    const double *v = nullptr;
};

inline InputView view_of(const InputData &d) {
    InputView w;
    w.m = d.m;
    w.nblk = d.nblk;
    w.bs = d.bs.data();
    w.c = d.c.data();
    w.nnz = (long long)d.v.size();
    w.mat = d.mat.data();
    w.blk = d.blk.data();
    w.i = d.i.data();
    w.j = d.j.data();
    w.v = d.v.data();
    return w;
}

struct Options {
    double tol = 1e-8;
    int maxit = 100;
    int verbose = 1;            // 0 quiet, 1 default log, 2.. diagnosis
    int lanczos_k = 30;
    double gamma_max = 0.99;
    double pivtol = 1e-14;
    double sigma_min = 0.0;
    double balance = 0.0;
    int sigma_rule = -1;
    int mixed = -1;             // FP32 Schur factor: -1 auto (m >= 1000), 0 never, 1 always
    int asm_prec = -1;          // Schur assembly: -1 auto (FP64), 0 FP64, 1 3xTF32, 2 FP64-accurate on the
                                // INT8 tensor cores (Ozaki slices)
    int late_prec = (5 << 8) | 2;   // 3xTF32 path: the assembly once the FP32-accurate M no longer serves (0 FP64,
                                // 2 Ozaki with 8 slices, FP64-accurate; (S << 8) | 2 with S = 4..7 slices, a
                                // preconditioner-grade M whose PCG residuals are taken with the FP64 operator,
                                // turned to 8 slices if its factor needs a shift or PCG misses)
    double mu_switch = 1e-4;    // 3xTF32 path: the factor goes to FP64 once scaled mu < mu_switch
    int mixed_shift = 0;        // 3xTF32 path: 1 keeps a shifted factor of M as the PCG preconditioner (slower
                                // on rand1000: 170 PCG steps per solve); 0 re-assembles in FP64
    int chunk = 0;              // constraints per assembly chunk (0: chosen by the block order)
    double timelimit = 0.0;
    double reg_ill = 0.0;
    int stall_win = 5;
    double red_acc = 1e-6;
    int known_feasible = 0;
    int device = 0;
    int sparse = -1;            // Schur factor: -1 auto (the reference's caps, solver.c:4014-4100), 0 dense,
                                // 1 supernodal sparse
    int init = 1;               // 0: SDPT3 start (start_sdpt3); 1: least-squares start (solver.c:13939-14198)
    int batch_mode = -1;        // bgpu_batch_solve: -1/1 lockstep when every problem has one block of order
                                // <= 64 (else concurrent), 0 concurrent per-problem solves
    int direction = -1;         // -1 auto (solver.c:13585-13591), 0 HKM, 1 NT
    int route = -1;             // Schur route per block: -1 auto (dense when the constraints average >= 2 % of
                                // n^2 entries, problem.c:1299), 0 row-product, 1 dense
    int hsd = -1;               // the self-dual embedding: -hsd 1, -nohsd 0, -1 the reference's rule
                                // (solver.c:13519-13560: the embedding first where its dense work is small)
    int batch_tune = 1;         // the lockstep batch's work-item autotuner (-batchtune 0|1)
    int lowrank = -1;           // the low-rank Schur route (-lowrank, problem.c:972): -1 where it is cheaper
                                // (every constraint of the block of low rank), 0 off, 1 wherever it applies
};

struct Timings {
    double setup = 0, schur = 0, chol = 0, dense = 0, step = 0, total = 0, read = 0;
};

struct ResultData {
    int status = -1;            // 0 optimal, 1 primal infeasible, 2 dual infeasible, 3 iteration limit,
                                // 4 numerical difficulties, 5 reduced accuracy, 6 time limit
    int exit_code = 0;
    int iters = 0;
    int direction = 0;          // the search direction taken: 0 HKM, 1 NT
    int embedding = 0;          // 1: solved by the self-dual embedding (Solver::run_hsd)
    int have_x = 0;
    int m = 0, nblk = 0;
    std::vector<int> bs;
    double pobj = 0, dobj = 0;  // <C,X>, b'y on the data as given
    double err[7] = {0, 0, 0, 0, 0, 0, 0};
    double time = 0;
    std::vector<double> y;
    std::vector<std::vector<double>> X, Z;
    Timings t;
    int nfloat = 0, nfactor = 0, pcg_iters = 0;
    double schur_flops = 0;     // algorithmic flops of the assembly GEMMs, summed over iterations
    double schur_time = 0;      // device time of the assemblies (s)
    double device_time = 0;     // CUDA-event time of the solve on the library's stream (s)
    double h2d_bytes = 0, d2h_bytes = 0;   // problem upload and result download
};

const char *status_string(int status);
int exit_code_of(int status);

// Parses command-line options (argv strings).  Returns 0 on success, 1 on a bad option.
int parse_options(int argc, const char *const *argv, Options &opt, std::string &err);

// Solves on the GPU; fills res.  Returns the exit code (0, 10-15) or a negative abort code.
int solve_problem(const InputView &in, const Options &opt, ResultData &res);

// A device arena for a batch worker: one allocation and one stream reused by every instance.
struct Arena {
    char *base = nullptr;
    size_t cap = 0, used = 0;
    size_t need = 0;      // set when an allocation did not fit: a lower bound of the bytes needed
    void *st = nullptr;   // cudaStream_t
    char *hbase = nullptr;   // pinned host memory for the loop's small reads
    size_t hcap = 0, hused = 0;
};
// Solves with the device memory and stream of the arena (no cudaMalloc / cudaFree, no device-wide
// synchronisation) and builds the host problem on the calling thread.  Returns BGPU_ERR_NOMEM
// (arena->need set) when the arena is too small; the caller grows it and calls again.
int solve_problem_arena(const InputView &in, const Options &opt, ResultData &res, Arena *arena);

// Solves `count` independent problems on `workers` host threads (0: one per host core), each
// with its own stream and arena, largest estimated work first.  get(p, in) fills problem p
// (false: bad problem, exit code 2); put(p, res, rc) receives its result.  Every instance runs
// the same code as solve_problem (quiet), so its result equals the stand-alone solve's.
// Returns 0, or 1 on bad options (err set).
// view(p, v) (optional) gives problem p in place, for the lockstep form's host build.
int solve_batch(int count, const std::vector<double> &work, const std::function<bool(int, InputData &)> &get,
                const std::function<void(int, ResultData &, int)> &put, const Options &opt, int workers,
                std::string &err, const std::function<bool(int, InputView &)> &view = nullptr);

// A batch of one-block problems (order <= 64) kept resident in HBM between lockstep solves.
struct BatchSession;
BatchSession *batch_session_create(int count, const std::function<bool(int, InputData &)> &get,
                                   const std::function<bool(int, InputView &)> &view, const Options &opt, int &rc);
int batch_session_solve(BatchSession *S, const std::function<void(int, ResultData &, int)> &put, int verbose);
void batch_session_destroy(BatchSession *S);

// A problem kept resident in HBM between solves (the benchmark's device-resident timing).
struct Session;
Session *session_create(const InputView &in, const Options &opt, std::string &err, int &rc);
int session_solve(Session *s, const Options &opt, ResultData &res);
void session_destroy(Session *s);

// Reads an SDPA sparse file (sdpa.cpp; the reference's read_sdpa, problem.c:426).  Returns 0, or
// 2 with a message in err.
int read_sdpa_file(const char *path, InputData &in, std::string &err);

// Output (the C API's brisk_set_output routes it).
void log_printf(int is_err, const char *fmt, ...);

}  // namespace bsolve
