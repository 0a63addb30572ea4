// The drop-in C interface: the exported brisk_* functions of the reference's libbrisk
// (capi.c:60-201, 520-535; version script libbrisk.map) for the semidefinite path, with the
// same argument meaning, return codes and accessor set.  Options are command-line strings
// (main.c:5846-5960 for the ones the Newton step reads); SDPA sparse files are read here.
#include "../../include/bgpu.h"
#include "../../include/brisk.h"
#include "solver.h"

#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace bsolve {
void set_print_hook(int (*f)(const char *, int));
}

struct BriskResult {
    bsolve::ResultData r;
    std::vector<const double *> Xp, Zp;
    std::string status_str;
};

namespace {
int g_out_mode = 0;
int (*g_out_cb)(const char *, int) = nullptr;
volatile int g_stop = 0;
int g_stop_owner = 0;

int capi_print(const char *s, int is_err) {
    if (g_out_mode == 2 && g_out_cb) return g_out_cb(s, is_err);
    if (g_out_mode == 1 && !is_err) return 0;
    fputs(s, is_err ? stderr : stdout);
    return 0;
}

void fill_result(BriskResult *res) {
    res->status_str = bsolve::status_string(res->r.status);
    res->Xp.assign(res->r.nblk, nullptr);
    res->Zp.assign(res->r.nblk, nullptr);
    for (int k = 0; k < res->r.nblk && k < (int)res->r.X.size(); k++) {
        res->Xp[k] = res->r.X[k].data();
        res->Zp[k] = res->r.Z[k].data();
    }
}

int run(const bsolve::InputView &in, int nopt, const char *const *opts, BriskResult *res) {
    bsolve::Options opt;
    std::string err;
    bsolve::set_print_hook(capi_print);
    if (bsolve::parse_options(nopt, opts, opt, err)) {
        bsolve::log_printf(1, "brisk: %s\n", err.c_str());
        fflush(stdout);
        return 1;
    }
    const int rc = bsolve::solve_problem(in, opt, res->r);
    fill_result(res);
    fflush(stdout);
    fflush(stderr);
    return rc;
}
}  // namespace

namespace bsolve {

static bool parse_double(const char *s, double &v) {
    if (!s) return false;
    char *e = nullptr;
    errno = 0;
    v = strtod(s, &e);
    return e != s && *e == 0 && errno == 0;
}
static bool parse_int(const char *s, int &v) {
    double d;
    if (!parse_double(s, d) || d != std::floor(d)) return false;
    v = (int)d;
    return true;
}

int parse_options(int argc, const char *const *argv, Options &opt, std::string &err) {
    bool tol_given = false;
    for (int i = 0; i < argc; i++) {
        const std::string a = argv[i] ? argv[i] : "";
        auto need = [&](const char *what) -> const char * {
            if (i + 1 >= argc) { err = std::string("option ") + a + " needs " + what; return nullptr; }
            return argv[++i];
        };
        if (a == "-tol") {
            const char *s = need("a number");
            if (!s || !parse_double(s, opt.tol) || !(opt.tol > 0)) { if (err.empty()) err = "bad -tol"; return 1; }
            tol_given = true;
        } else if (a == "-maxit") {
            const char *s = need("a number");
            if (!s || !parse_int(s, opt.maxit) || opt.maxit < 0) { if (err.empty()) err = "bad -maxit"; return 1; }
        } else if (a == "-lanczos") {
            const char *s = need("a number");
            if (!s || !parse_int(s, opt.lanczos_k) || opt.lanczos_k < 1) { if (err.empty()) err = "bad -lanczos"; return 1; }
        } else if (a == "-gmax") {
            const char *s = need("a number");
            if (!s || !parse_double(s, opt.gamma_max)) { if (err.empty()) err = "bad -gmax"; return 1; }
        } else if (a == "-pivtol") {
            const char *s = need("a number");
            if (!s || !parse_double(s, opt.pivtol)) { if (err.empty()) err = "bad -pivtol"; return 1; }
        } else if (a == "-regill") {
            const char *s = need("a number");
            if (!s || !parse_double(s, opt.reg_ill)) { if (err.empty()) err = "bad -regill"; return 1; }
        } else if (a == "-mixed") {
            const char *s = need("-1, 0 or 1");
            if (!s || !parse_int(s, opt.mixed)) { if (err.empty()) err = "bad -mixed"; return 1; }
        } else if (a == "-asmprec") {   // this build: the Schur assembly's precision
            const char *s = need("fp64, tf32x3, ozaki or ozaki4..ozaki7");
            if (!s) return 1;
            if (!strcmp(s, "fp64")) opt.asm_prec = 0;
            else if (!strcmp(s, "tf32x3")) opt.asm_prec = 1;
            else if (!strcmp(s, "ozaki") || !strcmp(s, "ozaki8")) opt.asm_prec = 2;
            else if (!strncmp(s, "ozaki", 5) && s[5] >= '4' && s[5] <= '7' && s[6] == 0) opt.asm_prec = ((s[5] - '0') << 8) | 2;
            else { err = "bad -asmprec (fp64, tf32x3, ozaki or ozaki4..ozaki7)"; return 1; }
        } else if (a == "-asmlate") {   // this build: the 3xTF32 path's late assembly
            const char *s = need("fp64, ozaki or ozaki4..ozaki7");
            if (!s) return 1;
            if (!strcmp(s, "fp64")) opt.late_prec = 0;
            else if (!strcmp(s, "ozaki") || !strcmp(s, "ozaki8")) opt.late_prec = 2;
            else if (!strncmp(s, "ozaki", 5) && s[5] >= '4' && s[5] <= '7' && s[6] == 0) opt.late_prec = ((s[5] - '0') << 8) | 2;
            else { err = "bad -asmlate (fp64, ozaki or ozaki4..ozaki7)"; return 1; }
        } else if (a == "-muswitch") {
            const char *s = need("a number");
            if (!s || !parse_double(s, opt.mu_switch)) { if (err.empty()) err = "bad -muswitch"; return 1; }
        } else if (a == "-mixedshift") {
            const char *s = need("0 or 1");
            if (!s || !parse_int(s, opt.mixed_shift) || opt.mixed_shift < 0 || opt.mixed_shift > 1) {
                if (err.empty()) err = "bad -mixedshift (0 or 1)";
                return 1;
            }
        } else if (a == "-schurchunk") {
            const char *s = need("8, 16, 32 or 64");
            if (!s || !parse_int(s, opt.chunk) || (opt.chunk != 8 && opt.chunk != 16 && opt.chunk != 32 && opt.chunk != 64)) {
                if (err.empty()) err = "bad -schurchunk";
                return 1;
            }
        } else if (a == "-device") {
            const char *s = need("a number");
            if (!s || !parse_int(s, opt.device)) { if (err.empty()) err = "bad -device"; return 1; }
        } else if (a == "-timelimit") {
            const char *s = need("a number");
            if (!s || !parse_double(s, opt.timelimit)) { if (err.empty()) err = "bad -timelimit"; return 1; }
        } else if (a == "-sigma") {
            const char *s = need("a number");
            if (!s || !parse_int(s, opt.sigma_rule)) { if (err.empty()) err = "bad -sigma"; return 1; }
        } else if (a == "-acc") {
            const char *s = need("low, medium or high");
            if (!s) return 1;
            if (!strcmp(s, "low")) { opt.tol = 1e-6; opt.red_acc = 1e-4; }
            else if (!strcmp(s, "high")) { opt.tol = 1e-10; opt.red_acc = 1e-6; }
            else if (!strcmp(s, "medium")) { opt.tol = 1e-8; opt.red_acc = 1e-6; }
            else { err = "bad -acc"; return 1; }
        } else if (a == "-dir") {
            const char *s = need("hkm, nt or auto");
            if (!s) return 1;
            if (!strcmp(s, "nt")) opt.direction = 1;
            else if (!strcmp(s, "hkm")) opt.direction = 0;
            else if (!strcmp(s, "auto")) opt.direction = -1;
            else { err = "-dir must be auto, hkm or nt"; return 1; }
        } else if (a == "-init") {
            const char *s = need("0 or 1");
            if (!s || !parse_int(s, opt.init) || opt.init < 0) { if (err.empty()) err = "bad -init"; return 1; }
        } else if (a == "-schurroute") {   // this build: the assembly route of every block
            const char *s = need("auto, row or dense");
            if (!s) return 1;
            if (!strcmp(s, "auto")) opt.route = -1;
            else if (!strcmp(s, "row")) opt.route = 0;
            else if (!strcmp(s, "dense")) opt.route = 1;
            else { err = "bad -schurroute (auto, row or dense)"; return 1; }
        } else if (a == "-batchtune") {   // this build: the lockstep batch's work-item autotuner
            const char *s = need("0 or 1");
            if (!s || !parse_int(s, opt.batch_tune) || opt.batch_tune < 0 || opt.batch_tune > 1) {
                if (err.empty()) err = "bad -batchtune (0 or 1)";
                return 1;
            }
        } else if (a == "-lowrank") {   // the reference's option: -1 auto, 0 off, 1 force
            const char *s = need("-1, 0 or 1");
            if (!s || !parse_int(s, opt.lowrank) || opt.lowrank < -1 || opt.lowrank > 1) {
                if (err.empty()) err = "bad -lowrank (-1 auto, 0 off, 1 force)";
                return 1;
            }
        } else if (a == "-q") {
            opt.verbose = 0;
        } else if (a == "-v") {
            opt.verbose = 2;
        } else if (a == "-vv" || a == "-vvv") {
            opt.verbose = 3;
        } else if (a == "-nohsd" || a == "-nofr" || a == "-feasible") {
            if (a == "-feasible") opt.known_feasible = 1;
            if (a == "-nohsd") opt.hsd = 0;
        } else if (a == "-hsd") {
            // a flag in the reference (OPTIONS.md: "-hsd | -nohsd"): the self-dual embedding
            opt.hsd = 1;
        } else if (a == "-corr" || a == "-chordal" || a == "-sym" || a == "-symalg" || a == "-deprows" ||
                   a == "-mixedfrac") {
            // options of the reference that change its method; this build solves the problem as
            // given with the infeasible-start predictor-corrector, so a value other than the one
            // that method already has is passed over with a note
            const char *s = need("a value");
            if (!s) return 1;
            const std::string v = s;
            const char *what = nullptr;
            if (a == "-corr" && v != "0") what = "centrality correctors are not run";
            else if (a == "-chordal" && v == "1") what = "no chordal decomposition is applied: the blocks are solved as given";
            else if (a == "-sym" && v != "none") what = "no symmetry reduction is applied";
            else if (a == "-symalg" && v != "0") what = "no block-algebra reduction is applied";
            else if (a == "-deprows" && v != "0") what = "dependent constraints are not removed";
            else if (a == "-mixedfrac") what = "the float-factor rule of this build does not use it";
            if (what) log_printf(1, "brisk: note: option %s %s: %s\n", a.c_str(), s, what);
        } else if (a == "-batchmode") {
            const char *s = need("lockstep or concurrent");
            if (!s) return 1;
            if (!strcmp(s, "lockstep")) opt.batch_mode = 1;
            else if (!strcmp(s, "concurrent")) opt.batch_mode = 0;
            else { err = "bad -batchmode (lockstep or concurrent)"; return 1; }
        } else if (a == "-sparse") {
            const char *s = need("-1, 0 or 1");
            if (!s || !parse_int(s, opt.sparse) || opt.sparse < -1 || opt.sparse > 1) {
                if (err.empty()) err = "bad -sparse (-1 auto, 0 dense, 1 sparse)";
                return 1;
            }
        } else if (a == "-threads" || a == "-caller") {
            // options of the reference that take a value and do not change the method (host
            // threads of its CPU solve; the calling language)
            if (!need("a value")) return 1;
        } else {
            // another of the reference's options (OPTIONS.md's table): its value, if it has one,
            // is the next argument when that is no option (a word, or a number such as -1)
            std::string shown = a;
            if (i + 1 < argc && argv[i + 1]) {
                const char *nx = argv[i + 1];
                const bool is_option = nx[0] == '-' && nx[1] != '\0' && !std::isdigit((unsigned char)nx[1]) && nx[1] != '.';
                if (!is_option) shown += std::string(" ") + argv[++i];
            }
            log_printf(1, "brisk: note: option %s is not used by the GPU Newton step (ignored)\n", shown.c_str());
        }
    }
    if (tol_given && 100.0 * opt.tol > opt.red_acc) opt.red_acc = 100.0 * opt.tol;
    return 0;
}

}  // namespace bsolve

// ---------------------------------------------------------------------------------------------
// exported interface
// ---------------------------------------------------------------------------------------------
// The caller's arrays as they are (nothing copied; build_problem skips the entries of value 0).
static bool make_view(int m, int nblk, const int *bs, const double *c, int64_t nnz, const int *mat, const int *blk,
                      const int *i, const int *j, const double *v, bsolve::InputView &in) {
    if (nnz < 0 || m < 0 || m > 100000000 || nblk <= 0 || !bs || (m > 0 && !c) ||
        (nnz > 0 && (!mat || !blk || !i || !j || !v))) {
        // the reference's message (problem.c, problem_from_sdpa_data)
        bsolve::log_printf(1, "brisk: invalid problem data (m = %d, %d blocks)\n", m, nblk);
        return false;
    }
    in.m = m;
    in.nblk = nblk;
    in.bs = bs;
    in.c = c;
    in.nnz = nnz;
    in.mat = mat;
    in.blk = blk;
    in.i = i;
    in.j = j;
    in.v = v;
    return true;
}

// The same numbers copied, zero values dropped (for callers that keep them past the call).
static bool make_input(int m, int nblk, const int *bs, const double *c, int64_t nnz, const int *mat, const int *blk,
                       const int *i, const int *j, const double *v, bsolve::InputData &in) {
    bsolve::InputView w;
    if (!make_view(m, nblk, bs, c, nnz, mat, blk, i, j, v, w)) return false;
    in.m = m;
    in.nblk = nblk;
    in.bs.assign(bs, bs + nblk);
    in.c.assign(c, c + m);
    in.mat.reserve(nnz);
    in.blk.reserve(nnz);
    in.i.reserve(nnz);
    in.j.reserve(nnz);
    in.v.reserve(nnz);
    for (int64_t q = 0; q < nnz; q++) {
        if (v[q] == 0) continue;
        in.mat.push_back(mat[q]);
        in.blk.push_back(blk[q]);
        in.i.push_back(i[q]);
        in.j.push_back(j[q]);
        in.v.push_back(v[q]);
    }
    return true;
}

extern "C" {

BRISK_API void brisk_set_output(int mode, int (*cb)(const char *s, int is_err)) {
    g_out_mode = mode;
    g_out_cb = cb;
}

BRISK_API const char *brisk_version(void) { return "1.7-b200"; }

BRISK_API BriskResult *brisk_result_new(void) {
    BriskResult *r = new (std::nothrow) BriskResult();
    if (r) r->r.status = -1;
    return r;
}
BRISK_API void brisk_result_delete(BriskResult *r) { delete r; }
BRISK_API int brisk_result_status(const BriskResult *r) { return r ? r->r.status : -1; }
BRISK_API const char *brisk_result_status_str(const BriskResult *r) {
    return r && r->r.status >= 0 ? r->status_str.c_str() : "NOT SOLVED";
}
BRISK_API int brisk_result_exit_code(const BriskResult *r) { return r ? r->r.exit_code : -1; }
BRISK_API int brisk_result_iterations(const BriskResult *r) { return r ? r->r.iters : 0; }
BRISK_API int brisk_result_m(const BriskResult *r) { return r ? r->r.m : 0; }
BRISK_API int brisk_result_nblk(const BriskResult *r) { return r ? r->r.nblk : 0; }
BRISK_API int brisk_result_blocksize(const BriskResult *r, int k) {
    return r && k >= 0 && k < (int)r->r.bs.size() ? r->r.bs[k] : 0;
}
BRISK_API double brisk_result_pobj(const BriskResult *r) { return r ? r->r.pobj : 0; }
BRISK_API double brisk_result_dobj(const BriskResult *r) { return r ? r->r.dobj : 0; }
BRISK_API double brisk_result_time(const BriskResult *r) { return r ? r->r.time : 0; }
BRISK_API int brisk_result_have_x(const BriskResult *r) { return r ? r->r.have_x : 0; }
BRISK_API void brisk_result_dimacs(const BriskResult *r, double *err) {
    for (int e = 0; e < 6; e++) err[e] = r ? r->r.err[e + 1] : 0;
}
BRISK_API const double *brisk_result_y(const BriskResult *r) { return r && !r->r.y.empty() ? r->r.y.data() : nullptr; }
BRISK_API const double *brisk_result_X(const BriskResult *r, int k) {
    return r && r->r.have_x && k >= 0 && k < (int)r->Xp.size() ? r->Xp[k] : nullptr;
}
BRISK_API const double *brisk_result_Z(const BriskResult *r, int k) {
    return r && k >= 0 && k < (int)r->Zp.size() ? r->Zp[k] : nullptr;
}
BRISK_API int brisk_result_bound(const BriskResult *r, double *out) {
    if (out) for (int q = 0; q < 6; q++) out[q] = 0;
    return 0;
}
BRISK_API int brisk_result_resolves(const BriskResult *r, double *t) {
    if (t) *t = 0;
    return 0;
}
BRISK_API const char *brisk_result_cause(const BriskResult *r) { return ""; }

BRISK_API void brisk_interrupt(void) { g_stop = 1; }
BRISK_API int brisk_interrupted(void) { return g_stop != 0; }
BRISK_API void brisk_clear_interrupt(void) { g_stop = 0; }
BRISK_API void brisk_set_interrupt_owner(int caller) { g_stop_owner = caller != 0; }

BRISK_API int brisk_solve_data(int m, int nblk, const int *bs, const double *c, int64_t nnz, const int *mat,
                               const int *blk, const int *i, const int *j, const double *v, int nopt,
                               const char *const *opts, BriskResult *res) {
    if (!res) return -1;
    res->r = bsolve::ResultData();
    if (!g_stop_owner) g_stop = 0;
    bsolve::InputView in;
    bsolve::set_print_hook(capi_print);
    if (!make_view(m, nblk, bs, c, nnz, mat, blk, i, j, v, in)) return 2;
    return run(in, nopt, opts, res);
}

BGPU_API int bgpu_batch_solve(int count, const int *m, const int *nblk, const int *bs, const double *c,
                              const int64_t *nnz, const int *mat, const int *blk, const int *i, const int *j,
                              const double *v, int nopt, const char *const *opts, int workers,
                              BriskResult *const *res, int *rc) {
    if (count < 0 || (count > 0 && (!m || !nblk || !bs || !nnz || !res || !rc))) return -1;
    std::vector<int64_t> boff(count + 1, 0), coff(count + 1, 0), eoff(count + 1, 0);
    std::vector<double> work(count, 0.0);
    for (int p = 0; p < count; p++) {
        if (!res[p] || nblk[p] < 0 || m[p] < 0 || nnz[p] < 0) return -1;
        boff[p + 1] = boff[p] + nblk[p];
        coff[p + 1] = coff[p] + m[p];
        eoff[p + 1] = eoff[p] + nnz[p];
        // assembly m (4 n^3 + 2 n^2 m) per block plus the factor m^3 / 3: the largest go first
        const double mm = m[p];
        double w = mm * mm * mm / 3.0;
        for (int k = 0; k < nblk[p]; k++) {
            const double n = std::fabs((double)bs[boff[p] + k]);
            w += mm * (4.0 * n * n * n + 2.0 * n * n * mm);
        }
        work[p] = w;
    }
    bsolve::Options opt;
    std::string err;
    bsolve::set_print_hook(capi_print);
    if (bsolve::parse_options(nopt, opts, opt, err)) {
        bsolve::log_printf(1, "brisk: %s\n", err.c_str());
        fflush(stdout);
        return 1;
    }
    auto get = [&](int p, bsolve::InputData &in) {
        const int64_t e = eoff[p];
        return make_input(m[p], nblk[p], bs + boff[p], c ? c + coff[p] : nullptr, nnz[p], mat ? mat + e : nullptr,
                          blk ? blk + e : nullptr, i ? i + e : nullptr, j ? j + e : nullptr, v ? v + e : nullptr, in);
    };
    auto put = [&](int p, bsolve::ResultData &r, int code) {
        res[p]->r = std::move(r);
        fill_result(res[p]);
        rc[p] = code;
    };
    auto view = [&](int p, bsolve::InputView &in) {
        const int64_t e = eoff[p];
        in.m = m[p];
        in.nblk = nblk[p];
        in.bs = bs + boff[p];
        in.c = c ? c + coff[p] : nullptr;
        in.nnz = nnz[p];
        in.mat = mat ? mat + e : nullptr;
        in.blk = blk ? blk + e : nullptr;
        in.i = i ? i + e : nullptr;
        in.j = j ? j + e : nullptr;
        in.v = v ? v + e : nullptr;
        return !(in.m < 0 || in.nblk <= 0 || (in.m > 0 && !in.c) ||
                 (in.nnz > 0 && (!in.mat || !in.blk || !in.i || !in.j || !in.v)));
    };
    return bsolve::solve_batch(count, work, get, put, opt, workers, err, view);
}

struct bgpu_batch {
    bsolve::BatchSession *s = nullptr;
    int count = 0;
    int verbose = 0;
};

BGPU_API bgpu_batch *bgpu_batch_create(int count, const int *m, const int *nblk, const int *bs, const double *c,
                                       const int64_t *nnz, const int *mat, const int *blk, const int *i, const int *j,
                                       const double *v, int nopt, const char *const *opts, int *rc) {
    int code = 0;
    if (count <= 0 || !m || !nblk || !bs || !nnz) code = -1;
    std::vector<int64_t> boff(count > 0 ? count + 1 : 1, 0), coff(boff), eoff(boff);
    for (int p = 0; !code && p < count; p++) {
        if (nblk[p] < 0 || m[p] < 0 || nnz[p] < 0) { code = -1; break; }
        boff[p + 1] = boff[p] + nblk[p];
        coff[p + 1] = coff[p] + m[p];
        eoff[p + 1] = eoff[p] + nnz[p];
    }
    bsolve::Options opt;
    std::string err;
    bsolve::set_print_hook(capi_print);
    if (!code && bsolve::parse_options(nopt, opts, opt, err)) {
        bsolve::log_printf(1, "brisk: %s\n", err.c_str());
        code = 1;
    }
    bgpu_batch *h = nullptr;
    if (!code) {
        auto view = [&](int p, bsolve::InputView &in) {
            const int64_t e = eoff[p];
            in.m = m[p];
            in.nblk = nblk[p];
            in.bs = bs + boff[p];
            in.c = c ? c + coff[p] : nullptr;
            in.nnz = nnz[p];
            in.mat = mat ? mat + e : nullptr;
            in.blk = blk ? blk + e : nullptr;
            in.i = i ? i + e : nullptr;
            in.j = j ? j + e : nullptr;
            in.v = v ? v + e : nullptr;
            return !(in.m < 0 || in.nblk <= 0 || (in.m > 0 && !in.c) ||
                     (in.nnz > 0 && (!in.mat || !in.blk || !in.i || !in.j || !in.v)));
        };
        int rc2 = 0;
        bsolve::BatchSession *s = bsolve::batch_session_create(count, nullptr, view, opt, rc2);
        if (s) {
            h = new bgpu_batch;
            h->s = s;
            h->count = count;
            h->verbose = opt.verbose;
        } else {
            code = rc2 ? rc2 : BGPU_ERR_UNSUPPORTED;
        }
    }
    if (rc) *rc = code;
    fflush(stdout);
    fflush(stderr);
    return h;
}

BGPU_API int bgpu_batch_run(bgpu_batch *h, BriskResult *const *res, int *rc) {
    if (!h || !res || !rc) return -1;
    for (int p = 0; p < h->count; p++)
        if (!res[p]) return -1;
    auto put = [&](int p, bsolve::ResultData &r, int code) {
        res[p]->r = std::move(r);
        fill_result(res[p]);
        rc[p] = code;
    };
    bsolve::set_print_hook(capi_print);
    const int code = bsolve::batch_session_solve(h->s, put, h->verbose);
    fflush(stdout);
    fflush(stderr);
    return code;
}

BGPU_API void bgpu_batch_destroy(bgpu_batch *h) {
    if (!h) return;
    bsolve::batch_session_destroy(h->s);
    delete h;
}

struct bgpu_session {
    bsolve::Session *s = nullptr;
};

BGPU_API bgpu_session *bgpu_session_create(int m, int nblk, const int *bs, const double *c, int64_t nnz,
                                           const int *mat, const int *blk, const int *i, const int *j,
                                           const double *v, int nopt, const char *const *opts, int *rc) {
    int code = 0;
    bsolve::InputView in;
    bsolve::Options opt;
    std::string err;
    bsolve::set_print_hook(capi_print);
    if (!make_view(m, nblk, bs, c, nnz, mat, blk, i, j, v, in)) code = 2;
    else if (bsolve::parse_options(nopt, opts, opt, err)) code = 1;
    bgpu_session *h = nullptr;
    if (!code) {
        bsolve::Session *s = bsolve::session_create(in, opt, err, code);
        if (s) {
            h = new bgpu_session;
            h->s = s;
        }
    }
    if (code) bsolve::log_printf(1, "brisk: %s\n", err.c_str());
    if (rc) *rc = code;
    return h;
}

BGPU_API int bgpu_session_solve(bgpu_session *h, int nopt, const char *const *opts, BriskResult *res) {
    if (!h || !res) return -1;
    bsolve::Options opt;
    std::string err;
    bsolve::set_print_hook(capi_print);
    if (bsolve::parse_options(nopt, opts, opt, err)) {
        bsolve::log_printf(1, "brisk: %s\n", err.c_str());
        return 1;
    }
    const int rc = bsolve::session_solve(h->s, opt, res->r);
    fill_result(res);
    fflush(stdout);
    return rc;
}

BGPU_API void bgpu_session_destroy(bgpu_session *h) {
    if (!h) return;
    bsolve::session_destroy(h->s);
    delete h;
}

BGPU_API int bgpu_result_measures(const BriskResult *r, double *out) {
    if (!r || !out) return BGPU_ERR_ARG;
    out[0] = r->r.device_time;
    out[1] = r->r.schur_time;
    out[2] = r->r.schur_flops;
    out[3] = r->r.h2d_bytes;
    out[4] = r->r.d2h_bytes;
    out[5] = r->r.iters;
    out[6] = r->r.nfloat;
    out[7] = r->r.pcg_iters;
    return BGPU_OK;
}

BRISK_API int brisk_solve_file(const char *fname, int nopt, const char *const *opts, BriskResult *res) {
    if (!res) return -1;
    res->r = bsolve::ResultData();
    if (!g_stop_owner) g_stop = 0;
    bsolve::InputData in;
    std::string err;
    bsolve::set_print_hook(capi_print);
    if (!fname || bsolve::read_sdpa_file(fname, in, err)) {
        bsolve::log_printf(1, "brisk: %s\n", err.c_str());
        return 2;
    }
    return run(bsolve::view_of(in), nopt, opts, res);
}

BGPU_API int bgpu_sdpa_read(const char *path, bgpu_sdpa *out) {
    if (!path || !out) return BGPU_ERR_ARG;
    *out = bgpu_sdpa();
    auto *in = new (std::nothrow) bsolve::InputData;
    if (!in) return BGPU_ERR_NOMEM;
    std::string err;
    bsolve::set_print_hook(capi_print);
    const int rc = bsolve::read_sdpa_file(path, *in, err);
    if (rc) {
        bsolve::log_printf(1, "brisk: %s\n", err.c_str());
        delete in;
        return rc;
    }
    out->m = in->m;
    out->nblk = in->nblk;
    out->nnz = (int64_t)in->v.size();
    out->bs = in->bs.data();
    out->c = in->c.data();
    out->mat = in->mat.data();
    out->blk = in->blk.data();
    out->i = in->i.data();
    out->j = in->j.data();
    out->v = in->v.data();
    out->owner = in;
    return 0;
}

BGPU_API void bgpu_sdpa_free(bgpu_sdpa *s) {
    if (!s) return;
    delete static_cast<bsolve::InputData *>(s->owner);
    *s = bgpu_sdpa();
}

}  // extern "C"
