// The lockstep batch: many independent problems with one SDP block of order <= 64 each (the
// uneven batch of bgpu_batch_solve) advanced together.  Each round is one interior-point
// iteration of every unfinished instance, with the scalar logic of Solver::run per instance
// (solver.c:14394-15188: sigma rule, gamma, refinement passes, catastrophe guard, try_step,
// stopping rules, best-iterate fallback) and every device step one launch over all instances:
//   - the constraints as packed rows P (m_k x n_k(n_k+1)/2, built once), A(.) and A'(.) from them;
//   - the Schur complements: Q = packed sym(X A_a Zi) for all (instance, constraint) work items,
//     then M_k = P_k Q_k' for every instance by one grouped DMMA GEMM (lower tiles only);
//   - one-CTA-per-instance Cholesky of D M D + reg I and triangular solves, PCG per instance;
//   - the small-block kernels (Z^-1, HKM products, exact lambda_min, Cholesky tests) over all
//     blocks, per-instance step lengths and per-instance coefficients in the element-wise work.
// Included by solver.cu inside its anonymous namespace (it uses the Solver's types).

class Lockstep {
  public:
    Lockstep(std::vector<HProblem> &probs, const Options &o) : Pb(probs), opt(o), B((int)probs.size()) {}
    ~Lockstep() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }
    void setup();
    void run(std::vector<ResultData> &res);

  private:
    std::vector<HProblem> &Pb;
    Options opt;
    int B;
    Gpu g;
    std::vector<int> n, m, t;
    std::vector<long long> boff, coff, moff, poff;
    long long Ntot2 = 0, mT = 0, MT = 0, PT = 0;
    int nmax = 1, mmax = 1;
    lockstep::Layout Ld;
    int *d_n = nullptr, *d_m = nullptr;
    long long *d_boff = nullptr, *d_coff = nullptr, *d_moff = nullptr, *d_poff = nullptr;
    DevArrays cat{};
    double *Ccat = nullptr, *Icat = nullptr, *Pp = nullptr, *Qp = nullptr, *Mm = nullptr, *Lf = nullptr, *Dsc = nullptr;
    double *d_reg = nullptr, *d_pmin = nullptr, *d_coef[4] = {nullptr, nullptr, nullptr, nullptr};
    int *d_info = nullptr, *d_list = nullptr, *d_flag = nullptr, *d_sinfo = nullptr;
    double *d_slam = nullptr;
    int2 *d_items = nullptr;
    int4 *d_tiles = nullptr;
    // the Q form's work-item size per block-order class (n <= 16, 32, 48, 64), 0 until tuned
    int class_item[4] = {0, 0, 0, 0};
    void tune_items(const std::vector<int> &L, const double *X, const double *Zi);
    static void class_items(const std::vector<int> &L, const std::vector<int> &n, const std::vector<int> &m, int c,
                            int item, std::vector<int2> &items);
    GemmGroup *d_groups = nullptr;
    long long max_items = 0, max_tiles = 0;
    double *dv_a = nullptr, *dv_b = nullptr, *d_dots = nullptr;
    const double **d_pa = nullptr, **d_pb = nullptr;
    double *h_a = nullptr, *h_b = nullptr, *h_dots = nullptr, *h_slam = nullptr, *h_pmin = nullptr;
    int *h_info = nullptr, *h_sinfo = nullptr;
    std::vector<std::pair<double *DevArrays::*, double **>> stab;
    std::vector<int> all;
    int *d_all = nullptr;   // 0 .. B-1
    int2 *d_aitems = nullptr, *d_titems = nullptr, *d_sitems = nullptr;   // A(.), A'(.), symv work items
    int n_aitems = 0, n_titems = 0;
    // per-instance factor state (schur_factor_)
    std::vector<double> reg, reg_ok, min_pivot;
    std::vector<char> reg_hint;
    std::vector<int> pcg_iters, nfactor;
    double schur_flops = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // the NT direction (every instance's block has order <= 64, so -dir auto takes NT): the scaling
    // G in NG, W = G G' in Zi, lam per instance from loff[k]
    bool nt = false;
    double *nlam = nullptr;
    long long *d_loff = nullptr;
    double **d_lamtab = nullptr;
    int *d_ntinfo = nullptr, *h_ntinfo = nullptr;
    void nt_toZ(double *DevArrays::*D, double *DevArrays::*out);     // out = sym(G' D G)
    void nt_fromS(double *DevArrays::*D, double *DevArrays::*out);   // out = sym(G D G')

  public:
    // wall time of the phases (s): start, assembly, factor, PCG, the rest of the loop, final measures;
    // of the set-up: allocations and tables, the upload of P
    double t_start = 0, t_asm = 0, t_fac = 0, t_pcg = 0, t_loop = 0, t_final = 0, t_alloc = 0, t_upload = 0;

  private:

    double **tab(double *DevArrays::*mem);
    void upload_list(const std::vector<int> &L);
    void set_coef(int i, const std::vector<double> &v);
    void mul(double *DevArrays::*A, double *DevArrays::*Bm, double *DevArrays::*C);
    void aop(const double *D, std::vector<double> &out);
    void atop(const std::vector<double> &y, double alpha, double beta, double *F);
    void segdots(int nq, const double *const *a, const double *const *b, std::vector<double> &out);
    void assemble(const std::vector<int> &L, const double *X, const double *Zi);
    void factor(const std::vector<int> &L, std::vector<int> &failed);
    void prec(const std::vector<int> &L, std::vector<double> &v);
    void symv(const std::vector<int> &L, const std::vector<double> &x, std::vector<double> &y);
    void pcg(const std::vector<int> &L, const std::vector<double> &rhs, std::vector<double> &x, double tol_rel);
    void maxstep(int primal, std::vector<double> &alpha);
    void try_step(int primal, const std::vector<int> &L, std::vector<double> &alpha, std::vector<char> &ok);
    void least_squares_start(std::vector<double> &y, std::vector<char> &started);
    void final_measures(const std::vector<double> &y, std::vector<ResultData> &res);
    double vdot(int k, const std::vector<double> &a, const std::vector<double> &b) const {
        double s = 0;
        for (long long i = coff[k]; i < coff[k + 1]; i++) s += a[i] * b[i];
        return s;
    }
};

void Lockstep::setup() {
    const double t_setup0 = wtime();
    CU(cudaSetDevice(opt.device));
    CU(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
    CU(cudaEventCreate(&ev0));
    CU(cudaEventCreate(&ev1));
    n.resize(B);
    m.resize(B);
    t.resize(B);
    boff.assign(B + 1, 0);
    coff.assign(B + 1, 0);
    moff.assign(B + 1, 0);
    poff.assign(B + 1, 0);
    for (int k = 0; k < B; k++) {
        n[k] = Pb[k].blk[0].n;
        m[k] = Pb[k].m;
        t[k] = n[k] * (n[k] + 1) / 2;
        boff[k + 1] = boff[k] + (long long)n[k] * n[k];
        coff[k + 1] = coff[k] + m[k];
        moff[k + 1] = moff[k] + (long long)m[k] * m[k];
        poff[k + 1] = poff[k] + (long long)m[k] * t[k];
        nmax = std::max(nmax, n[k]);
        mmax = std::max(mmax, m[k]);
    }
    Ntot2 = boff[B];
    mT = coff[B];
    MT = moff[B];
    PT = poff[B];
    all.resize(B);
    for (int k = 0; k < B; k++) all[k] = k;
    auto need = [](void *p) { if (!p) throw GpuFail{BGPU_ERR_NOMEM, __LINE__}; };
    d_n = g.alloc<int>(B);
    d_m = g.alloc<int>(B);
    d_boff = g.alloc<long long>(B + 1);
    d_coff = g.alloc<long long>(B + 1);
    d_moff = g.alloc<long long>(B + 1);
    d_poff = g.alloc<long long>(B + 1);
    need(d_n); need(d_m); need(d_boff); need(d_coff); need(d_moff); need(d_poff);
    for (double *DevArrays::*mem : kCatMembers) { cat.*mem = g.alloc<double>(Ntot2); need(cat.*mem); }
    nt = opt.direction != 0;   // auto: 15 n^3 <= 1e8 for every n <= 64 (solver.c:13585-13591)
    if (nt) {
        for (double *DevArrays::*mem : kNtMembers) { cat.*mem = g.alloc<double>(Ntot2); need(cat.*mem); }
        std::vector<long long> loff(B + 1, 0);
        for (int k = 0; k < B; k++) loff[k + 1] = loff[k] + n[k];
        nlam = g.alloc<double>(loff[B]);
        d_loff = g.alloc<long long>(B + 1);
        d_lamtab = g.alloc<double *>(B);
        d_ntinfo = g.alloc<int>(B);
        h_ntinfo = g.host_alloc<int>(B);
        need(nlam); need(d_loff); need(d_lamtab); need(d_ntinfo); need(h_ntinfo);
        std::vector<double *> lp(B);
        for (int k = 0; k < B; k++) lp[k] = nlam + loff[k];
        CU(cudaMemcpyAsync(d_loff, loff.data(), sizeof(long long) * (B + 1), cudaMemcpyHostToDevice, g.st));
        CU(cudaMemcpyAsync(d_lamtab, lp.data(), sizeof(double *) * B, cudaMemcpyHostToDevice, g.st));
        CU(cudaStreamSynchronize(g.st));
    }
    Ccat = g.alloc<double>(Ntot2);
    Icat = g.alloc<double>(Ntot2);
    Pp = g.alloc<double>(PT);
    Qp = g.alloc<double>(PT);
    Mm = g.alloc<double>(MT);
    Lf = g.alloc<double>(MT);
    Dsc = g.alloc<double>(mT);
    dv_a = g.alloc<double>(mT);
    dv_b = g.alloc<double>(mT);
    need(Ccat); need(Icat); need(Pp); need(Qp); need(Mm); need(Lf); need(Dsc); need(dv_a); need(dv_b);
    d_reg = g.alloc<double>(B);
    d_pmin = g.alloc<double>(B);
    d_info = g.alloc<int>(B);
    d_list = g.alloc<int>(B);
    d_all = g.alloc<int>(B);
    d_flag = g.alloc<int>(B);
    d_sinfo = g.alloc<int>(B);
    d_slam = g.alloc<double>(B);
    d_dots = g.alloc<double>((size_t)B * 8);
    d_pa = (const double **)g.alloc<double *>(8);
    d_pb = (const double **)g.alloc<double *>(8);
    need(d_reg); need(d_pmin); need(d_info); need(d_list); need(d_all); need(d_flag); need(d_sinfo); need(d_slam); need(d_dots);
    need(d_pa); need(d_pb);
    for (int i = 0; i < 4; i++) { d_coef[i] = g.alloc<double>(B); need(d_coef[i]); }
    for (int k = 0; k < B; k++) max_items += (m[k] + lockstep::ITEM_MIN - 1) / lockstep::ITEM_MIN;
    const int TR = gemm_grouped_tile_rows();
    for (int k = 0; k < B; k++) max_tiles += (long long)ceil_div(m[k], TR) * ceil_div(m[k], 64);
    {   // the work items of A(.) (RI rows) and A'(.) (256 packed entries) over all instances
        std::vector<int2> ai, ti;
        for (int k = 0; k < B; k++) {
            for (int r0 = 0; r0 < m[k]; r0 += lockstep::RI) ai.push_back(make_int2(k, r0));
            for (int u0 = 0; u0 < t[k]; u0 += 256) ti.push_back(make_int2(k, u0));
        }
        n_aitems = (int)ai.size();
        n_titems = (int)ti.size();
        d_aitems = g.alloc<int2>(ai.size());
        d_titems = g.alloc<int2>(ti.size());
        d_sitems = g.alloc<int2>(ai.size());
        need(d_aitems); need(d_titems); need(d_sitems);
        CU(cudaMemcpyAsync(d_aitems, ai.data(), sizeof(int2) * ai.size(), cudaMemcpyHostToDevice, g.st));
        CU(cudaMemcpyAsync(d_titems, ti.data(), sizeof(int2) * ti.size(), cudaMemcpyHostToDevice, g.st));
        CU(cudaStreamSynchronize(g.st));
    }
    d_items = g.alloc<int2>(max_items);
    d_tiles = g.alloc<int4>(max_tiles);
    d_groups = g.alloc<GemmGroup>(B);
    need(d_items); need(d_tiles); need(d_groups);
    h_a = g.host_alloc<double>(mT);
    h_b = g.host_alloc<double>(mT);
    h_dots = g.host_alloc<double>((size_t)B * 8);
    h_slam = g.host_alloc<double>(B);
    h_pmin = g.host_alloc<double>(B);
    h_info = g.host_alloc<int>(B);
    h_sinfo = g.host_alloc<int>(B);
    need(h_a); need(h_b); need(h_dots); need(h_slam); need(h_pmin); need(h_info); need(h_sinfo);
    CU(cudaMemcpyAsync(d_all, all.data(), sizeof(int) * B, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_n, n.data(), sizeof(int) * B, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_m, m.data(), sizeof(int) * B, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_boff, boff.data(), sizeof(long long) * (B + 1), cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_coff, coff.data(), sizeof(long long) * (B + 1), cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_moff, moff.data(), sizeof(long long) * (B + 1), cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_poff, poff.data(), sizeof(long long) * (B + 1), cudaMemcpyHostToDevice, g.st));
    Ld.B = B;
    Ld.n = d_n;
    Ld.m = d_m;
    Ld.boff = d_boff;
    Ld.coff = d_coff;
    Ld.moff = d_moff;
    Ld.poff = d_poff;
    // the grouped GEMM's groups: M_k = P_k Q_k' (m_k x m_k, K = t_k)
    {
        std::vector<GemmGroup> gr(B);
        for (int k = 0; k < B; k++) {
            gr[k].A = Pp + poff[k];
            gr[k].B = Qp + poff[k];
            gr[k].C = Mm + moff[k];
            gr[k].M = gr[k].N = m[k];
            gr[k].K = t[k];
            gr[k].lda = gr[k].ldb = t[k];
            gr[k].ldc = m[k];
        }
        CU(cudaMemcpyAsync(d_groups, gr.data(), sizeof(GemmGroup) * B, cudaMemcpyHostToDevice, g.st));
        CU(cudaStreamSynchronize(g.st));
    }
    t_alloc = wtime() - t_setup0;
    // P (the packed constraints, built with the problems) and C, uploaded.  P (gigabytes for
    // thousands of instances) goes through two pinned 64 MB buffers in turn: the host threads fill
    // one with the next instances' rows while the copy engine drains the other.
    std::vector<double> Ch(Ntot2, 0.0);
    {
        for (int k = 0; k < B; k++) {
            if ((long long)Pb[k].Cdense.size() != (long long)n[k] * n[k]) throw GpuFail{BGPU_ERR_ARG, __LINE__};
            std::copy(Pb[k].Cdense.begin(), Pb[k].Cdense.end(), Ch.begin() + boff[k]);
            if ((long long)Pb[k].packed.size() != (long long)m[k] * t[k]) throw GpuFail{BGPU_ERR_ARG, __LINE__};
        }
        constexpr long long RING = (64LL << 20) / (long long)sizeof(double);   // doubles per buffer
        double *ring[2] = {g.host_alloc<double>(RING), g.host_alloc<double>(RING)};
        need(ring[0]); need(ring[1]);
        cudaEvent_t done[2];
        CU(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming));
        bool used[2] = {false, false};
        int k = 0, buf = 0;
        long long kpos = 0;   // doubles of instance k already staged
        while (k < B) {
            if (used[buf]) CU(cudaEventSynchronize(done[buf]));
            // the pieces of this buffer: (instance, first double, count), in P's order
            struct Piece { int k; long long from, cnt, at; };
            std::vector<Piece> pieces;
            long long fill = 0;
            const long long first = poff[k] + kpos;
            while (k < B && fill < RING) {
                const long long left = (long long)Pb[k].packed.size() - kpos;
                const long long take = std::min(left, RING - fill);
                for (long long c = 0; c < take; c += (1LL << 17))   // 1 MB pieces for the threads
                    pieces.push_back({k, kpos + c, std::min(take - c, 1LL << 17), fill + c});
                fill += take;
                kpos += take;
                if (kpos == (long long)Pb[k].packed.size()) { k++; kpos = 0; }
            }
            double *dst = ring[buf];
            parallel_for((long long)pieces.size(), [&](long long q) {
                const Piece &pc = pieces[q];
                std::memcpy(dst + pc.at, Pb[pc.k].packed.data() + pc.from, sizeof(double) * pc.cnt);
            });
            if (fill > 0) {
                CU(cudaMemcpyAsync(Pp + first, dst, sizeof(double) * fill, cudaMemcpyHostToDevice, g.st));
                CU(cudaEventRecord(done[buf], g.st));
                used[buf] = true;
            }
            buf ^= 1;
        }
        CU(cudaStreamSynchronize(g.st));
        cudaEventDestroy(done[0]);
        cudaEventDestroy(done[1]);
        t_upload = wtime() - t_setup0 - t_alloc;
        CU(cudaMemcpyAsync(Ccat, Ch.data(), sizeof(double) * Ntot2, cudaMemcpyHostToDevice, g.st));
        std::vector<double> ones(B, 1.0);
        CU(cudaMemcpyAsync(d_coef[0], ones.data(), sizeof(double) * B, cudaMemcpyHostToDevice, g.st));
        RC(ew_scaled_identity_blocks(g.st, B, d_n, d_boff, Ntot2, d_coef[0], nullptr, Icat));
        CU(cudaStreamSynchronize(g.st));
    }
    reg.assign(B, 0.0);
    reg_ok.assign(B, 0.0);
    min_pivot.assign(B, 1.0);
    reg_hint.assign(B, 0);
    pcg_iters.assign(B, 0);
    nfactor.assign(B, 0);
}

double **Lockstep::tab(double *DevArrays::*mem) {
    for (auto &e : stab)
        if (e.first == mem) return e.second;
    std::vector<double *> ptrs(B);
    for (int k = 0; k < B; k++) ptrs[k] = cat.*mem + boff[k];
    double **d = g.alloc<double *>(B);
    if (!d) throw GpuFail{BGPU_ERR_NOMEM, __LINE__};
    CU(cudaMemcpyAsync(d, ptrs.data(), sizeof(double *) * B, cudaMemcpyHostToDevice, g.st));
    CU(cudaStreamSynchronize(g.st));
    stab.push_back({mem, d});
    return d;
}

void Lockstep::upload_list(const std::vector<int> &L) {
    CU(cudaMemcpyAsync(d_list, L.data(), sizeof(int) * L.size(), cudaMemcpyHostToDevice, g.st));
    CU(cudaStreamSynchronize(g.st));
}

void Lockstep::set_coef(int i, const std::vector<double> &v) {
    CU(cudaMemcpyAsync(d_coef[i], v.data(), sizeof(double) * B, cudaMemcpyHostToDevice, g.st));
    CU(cudaStreamSynchronize(g.st));   // v is pageable host memory the caller may change next
}

// nt_toZ / nt_fromS (solver.c:7990-8008, 8051-8068) for every instance (T is the scratch)
void Lockstep::nt_toZ(double *DevArrays::*D, double *DevArrays::*out) {
    RC(small_gemm(g.st, B, d_n, 0, 0, 1.0, (const double *const *)tab(D), (const double *const *)tab(&DevArrays::NG),
                  0.0, tab(&DevArrays::T), 0));
    RC(small_gemm(g.st, B, d_n, 1, 0, 1.0, (const double *const *)tab(&DevArrays::NG),
                  (const double *const *)tab(&DevArrays::T), 0.0, tab(out), 1));
}
void Lockstep::nt_fromS(double *DevArrays::*D, double *DevArrays::*out) {
    RC(small_gemm(g.st, B, d_n, 0, 0, 1.0, (const double *const *)tab(&DevArrays::NG), (const double *const *)tab(D),
                  0.0, tab(&DevArrays::T), 0));
    RC(small_gemm(g.st, B, d_n, 0, 1, 1.0, (const double *const *)tab(&DevArrays::T),
                  (const double *const *)tab(&DevArrays::NG), 0.0, tab(out), 1));
}

void Lockstep::mul(double *DevArrays::*A, double *DevArrays::*Bm, double *DevArrays::*C) {
    RC(small_gemm(g.st, B, d_n, 0, 0, 1.0, (const double *const *)tab(A), (const double *const *)tab(Bm), 0.0, tab(C),
                  0));
}

void Lockstep::aop(const double *D, std::vector<double> &out) {
    RC(lockstep::aop_packed(g.st, Ld, d_aitems, n_aitems, nmax, Pp, D, dv_a));
    CU(cudaMemcpyAsync(h_a, dv_a, sizeof(double) * mT, cudaMemcpyDeviceToHost, g.st));
    CU(cudaStreamSynchronize(g.st));
    out.assign(h_a, h_a + mT);
}

void Lockstep::atop(const std::vector<double> &y, double alpha, double beta, double *F) {
    std::copy(y.begin(), y.end(), h_a);
    CU(cudaMemcpyAsync(dv_a, h_a, sizeof(double) * mT, cudaMemcpyHostToDevice, g.st));
    RC(lockstep::atop_packed(g.st, Ld, d_titems, n_titems, Pp, dv_a, alpha, beta, F));
    CU(cudaStreamSynchronize(g.st));   // h_a is reused by the next call
}

void Lockstep::segdots(int nq, const double *const *a, const double *const *b, std::vector<double> &out) {
    CU(cudaMemcpyAsync(d_pa, a, sizeof(double *) * nq, cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_pb, b, sizeof(double *) * nq, cudaMemcpyHostToDevice, g.st));
    RC(lockstep::seg_dots(g.st, B, d_boff, nq, d_pa, d_pb, d_dots));
    CU(cudaMemcpyAsync(h_dots, d_dots, sizeof(double) * B * nq, cudaMemcpyDeviceToHost, g.st));
    CU(cudaStreamSynchronize(g.st));
    out.assign(h_dots, h_dots + (size_t)B * nq);
}

// The block-order classes of the Q form (a launch's shared memory is sized by its largest n, so
// the small classes run several CTAs per SM): class c holds the instances with cls_max[c-1] < n
// <= cls_max[c].
static const int cls_max[4] = {16, 32, 48, 64};

void Lockstep::class_items(const std::vector<int> &L, const std::vector<int> &n, const std::vector<int> &m, int c,
                           int item, std::vector<int2> &items) {
    for (int k : L)
        if (n[k] <= cls_max[c] && (c == 0 || n[k] > cls_max[c - 1]))
            for (int a0 = 0; a0 < m[k]; a0 += item) items.push_back(make_int2(k, a0));
}

// The autotuner of the batch's work-item shape: for each block-order class, the number of
// constraints one CTA of the Q form takes (its X and Zi loaded once for them) is timed on this
// batch's own data, every candidate in turn (CUDA events on the solve's stream, after one
// untimed launch of each), and the fastest kept.  Few constraints a CTA give more CTAs (small
// classes, few instances); many amortise the loads of X and Zi (large classes).  The choice is
// cached for the process by (device, class, the class's constraint count to a power of two), so
// later batches of the same shape skip the timing.  Every candidate writes the same Q.
void Lockstep::tune_items(const std::vector<int> &L, const double *X, const double *Zi) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int>, int> cache;
    int dev = 0;
    CU(cudaGetDevice(&dev));
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    std::string note;
    for (int c = 0; c < 4; c++) {
        long long cons = 0;
        for (int k : L)
            if (n[k] <= cls_max[c] && (c == 0 || n[k] > cls_max[c - 1])) cons += m[k];
        if (cons == 0) { class_item[c] = lockstep::ITEM; continue; }
        int bucket = 0;
        while ((1LL << bucket) < cons) bucket++;
        const auto key = std::make_tuple(dev, c, bucket);
        {
            std::lock_guard<std::mutex> lk(mu);
            auto it = cache.find(key);
            if (it != cache.end()) { class_item[c] = it->second; continue; }
        }
        int best = lockstep::ITEM;
        float best_ms = 1e30f;
        char buf[160];
        int w = snprintf(buf, sizeof buf, " n<=%d:", cls_max[c]);
        for (int item : lockstep::ITEM_CANDIDATES) {
            std::vector<int2> items;
            class_items(L, n, m, c, item, items);
            CU(cudaMemcpyAsync(d_items, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice, g.st));
            float ms = 0;
            for (int rep = 0; rep < 2; rep++) {   // the first launch untimed
                CU(cudaEventRecord(e0, g.st));
                RC(lockstep::form_q(g.st, Ld, d_items, (int)items.size(), cls_max[c], item, Pp, X, Zi, Qp));
                CU(cudaEventRecord(e1, g.st));
                CU(cudaEventSynchronize(e1));
                CU(cudaEventElapsedTime(&ms, e0, e1));
            }
            if (w < (int)sizeof buf) w += snprintf(buf + w, sizeof buf - w, " %d %.3f ms", item, ms);
            if (ms < best_ms) { best_ms = ms; best = item; }
        }
        class_item[c] = best;
        note += buf;
        std::lock_guard<std::mutex> lk(mu);
        cache[key] = best;
    }
    CU(cudaEventDestroy(e0));
    CU(cudaEventDestroy(e1));
    if (opt.verbose > 1 && !note.empty())
        log_printf(0, "   [batch work items tuned (constraints a CTA, Q form time):%s; taken: %d %d %d %d]\n", note.c_str(),
                   class_item[0], class_item[1], class_item[2], class_item[3]);
}

void Lockstep::assemble(const std::vector<int> &L, const double *X, const double *Zi) {
    if (L.empty()) return;
    const double t0 = wtime();
    if (class_item[0] == 0) {
        if (opt.batch_tune) tune_items(L, X, Zi);
        else for (int &c : class_item) c = lockstep::ITEM;
    }
    std::vector<int2> items;
    std::vector<int> cls_start(5, 0);
    std::vector<int4> tiles;
    const int TR = gemm_grouped_tile_rows();
    for (int c = 0; c < 4; c++) {
        cls_start[c] = (int)items.size();
        class_items(L, n, m, c, class_item[c], items);
    }
    cls_start[4] = (int)items.size();
    for (int k : L) {
        for (int ti = 0; ti < ceil_div(m[k], TR); ti++)
            for (int tj = 0; tj < ceil_div(m[k], 64); tj++)
                if (ti * TR + TR - 1 >= tj * 64) tiles.push_back(make_int4(k, ti, tj, 0));
        schur_flops += (double)m[k] * (4.0 * n[k] * n[k] * n[k] + 2.0 * n[k] * n[k] * m[k]);
    }
    CU(cudaMemcpyAsync(d_items, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice, g.st));
    CU(cudaMemcpyAsync(d_tiles, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice, g.st));
    for (int c = 0; c < 4; c++)
        RC(lockstep::form_q(g.st, Ld, d_items + cls_start[c], cls_start[c + 1] - cls_start[c], cls_max[c],
                            class_item[c], Pp, X, Zi, Qp));
    RC(gemm_f64_grouped(g.st, (int)tiles.size(), d_tiles, d_groups, 1.0, 0.0));
    upload_list(L);
    RC(lockstep::mirror(g.st, Ld, d_list, (int)L.size(), Mm));
    CU(cudaStreamSynchronize(g.st));
    t_asm += wtime() - t0;
}

// schur_factor_ (solver.c:5296-5421), FP64, per instance: the regularization ladder of Solver::factor
void Lockstep::factor(const std::vector<int> &L, std::vector<int> &failed) {
    const double t0 = wtime();
    const double ulp = 2.220446049250313e-16;
    std::vector<int> todo = L;
    std::vector<double> r(B, 0.0);
    for (int k : L) {
        nfactor[k]++;
        const double floor_k = opt.reg_ill > 0 ? opt.reg_ill : std::max(1e-15, (double)m[k] * ulp);
        r[k] = reg_hint[k] ? std::max(floor_k, 0.01 * reg_ok[k]) : 0.0;
    }
    failed.clear();
    for (int attempt = 0; attempt < 10 && !todo.empty(); attempt++) {
        CU(cudaMemcpyAsync(d_reg, r.data(), sizeof(double) * B, cudaMemcpyHostToDevice, g.st));
        upload_list(todo);
        RC(lockstep::chol(g.st, Ld, d_list, (int)todo.size(), Mm, d_reg, Dsc, Lf, d_info, d_pmin));
        CU(cudaMemcpyAsync(h_info, d_info, sizeof(int) * B, cudaMemcpyDeviceToHost, g.st));
        CU(cudaMemcpyAsync(h_pmin, d_pmin, sizeof(double) * B, cudaMemcpyDeviceToHost, g.st));
        CU(cudaStreamSynchronize(g.st));
        std::vector<int> again;
        for (int k : todo) {
            const double floor_k = opt.reg_ill > 0 ? opt.reg_ill : std::max(1e-15, (double)m[k] * ulp);
            const double first_k = opt.reg_ill > 0 ? 1e-13 : std::max(1e-15, (double)m[k] * ulp);
            if (h_info[k] == 0) {
                const double pmin = std::min(h_pmin[k], 1.0);
                if (pmin >= opt.pivtol || r[k] >= floor_k) {
                    reg[k] = r[k];
                    min_pivot[k] = pmin;
                    reg_hint[k] = r[k] > 0;
                    reg_ok[k] = r[k];
                    continue;
                }
                r[k] = std::max(floor_k, r[k] * 100);
            } else {
                r[k] = (r[k] == 0) ? first_k : r[k] * 100;
            }
            again.push_back(k);
        }
        todo.swap(again);
    }
    failed = todo;
    t_fac += wtime() - t0;
}

void Lockstep::prec(const std::vector<int> &L, std::vector<double> &v) {
    std::copy(v.begin(), v.end(), h_b);
    CU(cudaMemcpyAsync(dv_b, h_b, sizeof(double) * mT, cudaMemcpyHostToDevice, g.st));
    upload_list(L);
    RC(lockstep::prec(g.st, Ld, d_list, (int)L.size(), mmax, Lf, Dsc, dv_b));
    CU(cudaMemcpyAsync(h_b, dv_b, sizeof(double) * mT, cudaMemcpyDeviceToHost, g.st));
    CU(cudaStreamSynchronize(g.st));
    for (int k : L) std::copy(h_b + coff[k], h_b + coff[k + 1], v.begin() + coff[k]);
}

void Lockstep::symv(const std::vector<int> &L, const std::vector<double> &x, std::vector<double> &y) {
    std::copy(x.begin(), x.end(), h_b);
    CU(cudaMemcpyAsync(dv_b, h_b, sizeof(double) * mT, cudaMemcpyHostToDevice, g.st));
    std::vector<int2> si;
    for (int k : L)
        for (int c0 = 0; c0 < m[k]; c0 += lockstep::RI) si.push_back(make_int2(k, c0));
    CU(cudaMemcpyAsync(d_sitems, si.data(), sizeof(int2) * si.size(), cudaMemcpyHostToDevice, g.st));
    RC(lockstep::symv(g.st, Ld, d_sitems, (int)si.size(), Mm, dv_b, dv_a));
    CU(cudaMemcpyAsync(h_a, dv_a, sizeof(double) * mT, cudaMemcpyDeviceToHost, g.st));
    CU(cudaStreamSynchronize(g.st));
    y.resize(mT);
    for (int k : L) std::copy(h_a + coff[k], h_a + coff[k + 1], y.begin() + coff[k]);
}

// schur_solve_ (solver.c:5483-5621) per instance: PCG on M x = rhs with the exact FP64 factor
void Lockstep::pcg(const std::vector<int> &L, const std::vector<double> &rhs, std::vector<double> &x, double tol_rel) {
    const double t0 = wtime();
    struct Acc {
        double &t, t0;
        ~Acc() { t += wtime() - t0; }
    } acc{t_pcg, t0};
    x.assign(mT, 0.0);
    std::vector<int> run;
    std::vector<double> nb(B, 0.0), tol(B, 0.0), best(B, 0.0), rz(B, 0.0), nr(B, 0.0);
    std::vector<int> stall(B, 0), maxit(B, 10), used(B, 0);
    for (int k : L) {
        double s = 0;
        for (long long i = coff[k]; i < coff[k + 1]; i++) s += rhs[i] * rhs[i];
        nb[k] = std::sqrt(s);
        if (nb[k] > 0) run.push_back(k);
    }
    if (run.empty()) return;
    std::vector<double> r(mT, 0.0), z, p, q, xb, Mx;
    for (int k : run) std::copy(rhs.begin() + coff[k], rhs.begin() + coff[k + 1], x.begin() + coff[k]);
    prec(run, x);
    symv(run, x, Mx);
    std::vector<int> go;
    for (int k : run) {
        double s = 0;
        for (long long i = coff[k]; i < coff[k + 1]; i++) {
            r[i] = rhs[i] - Mx[i];
            s += r[i] * r[i];
        }
        nr[k] = std::sqrt(s);
        tol[k] = std::max(tol_rel, 1e-13) * nb[k];
        if (nr[k] > tol[k]) go.push_back(k);
        best[k] = nr[k];
        maxit[k] = reg[k] > 0 ? 50 : 10;
    }
    if (go.empty()) return;
    xb = x;
    z = r;
    prec(go, z);
    p = z;
    for (int k : go) rz[k] = vdot(k, r, z);
    const double sgain = 0.9;
    const int smax = 4;
    for (int it = 0; it < 50 && !go.empty(); it++) {
        symv(go, p, q);
        std::vector<int> cont;
        for (int k : go) {
            const double pq = vdot(k, p, q);
            if (!(pq > 0)) continue;
            const double a = rz[k] / pq;
            double s = 0;
            for (long long i = coff[k]; i < coff[k + 1]; i++) {
                x[i] += a * p[i];
                r[i] -= a * q[i];
                s += r[i] * r[i];
            }
            pcg_iters[k]++;
            used[k]++;
            nr[k] = std::sqrt(s);
            if (nr[k] < best[k]) {
                stall[k] = (nr[k] > sgain * best[k]) ? stall[k] + 1 : 0;
                best[k] = nr[k];
                std::copy(x.begin() + coff[k], x.begin() + coff[k + 1], xb.begin() + coff[k]);
            } else stall[k]++;
            if (nr[k] <= tol[k] || stall[k] >= smax || used[k] >= maxit[k]) continue;
            cont.push_back(k);
        }
        go.swap(cont);
        if (go.empty()) break;
        for (int k : go) std::copy(r.begin() + coff[k], r.begin() + coff[k + 1], z.begin() + coff[k]);
        prec(go, z);
        for (int k : go) {
            const double rz2 = vdot(k, r, z);
            const double beta = rz2 / rz[k];
            rz[k] = rz2;
            for (long long i = coff[k]; i < coff[k + 1]; i++) p[i] = z[i] + beta * p[i];
        }
    }
    for (int k : run) std::copy(xb.begin() + coff[k], xb.begin() + coff[k + 1], x.begin() + coff[k]);
}

// sdp_maxstep_lam for small blocks: the exact lambda_min of Li dV Li' per instance
void Lockstep::maxstep(int primal, std::vector<double> &alpha) {
    RC(small_lammin(g.st, B, d_n, (const double *const *)tab(primal ? &DevArrays::LiX : &DevArrays::LiZ),
                    (const double *const *)tab(primal ? &DevArrays::dX : &DevArrays::dZ), d_slam));
    CU(cudaMemcpyAsync(h_slam, d_slam, sizeof(double) * B, cudaMemcpyDeviceToHost, g.st));
    CU(cudaStreamSynchronize(g.st));
    alpha.assign(B, 1e30);
    for (int k = 0; k < B; k++) {
        const double lam = h_slam[k];
        double ak = (lam <= -1e299) ? 0.0 : (lam >= 0 ? 1e30 : -1.0 / lam);
        if (!std::isfinite(ak) && !(ak > 0)) ak = 0.0;
        alpha[k] = ak;
    }
}

// try_step (solver.c:6393-6447) per instance: V += alpha dV with a Cholesky test, alpha *= 0.8
void Lockstep::try_step(int primal, const std::vector<int> &L, std::vector<double> &alpha, std::vector<char> &ok) {
    std::vector<double> a(B, 0.0), stepped(B, 0.0), inc(B, 0.0);
    std::vector<int> tries(B, 0);
    ok.assign(B, 0);
    std::vector<int> todo = L;
    for (int k : L) a[k] = alpha[k];
    double *DevArrays::*V = primal ? &DevArrays::X : &DevArrays::Z;
    double *DevArrays::*dV = primal ? &DevArrays::dX : &DevArrays::dZ;
    double *DevArrays::*Lm_ = primal ? &DevArrays::LX : &DevArrays::LZ;
    double *DevArrays::*Li = primal ? &DevArrays::LiX : &DevArrays::LiZ;
    while (!todo.empty()) {
        std::fill(inc.begin(), inc.end(), 0.0);
        for (int k : todo) {
            inc[k] = a[k] - stepped[k];
            stepped[k] = a[k];
        }
        set_coef(3, inc);
        RC(ew_step_copy_coef(g.st, B, d_boff, Ntot2, d_coef[3], cat.*dV, cat.*V, cat.*Lm_));
        RC(small_chol_inv(g.st, B, d_n, tab(Lm_), tab(Lm_), tab(Li), d_sinfo));
        CU(cudaMemcpyAsync(h_sinfo, d_sinfo, sizeof(int) * B, cudaMemcpyDeviceToHost, g.st));
        CU(cudaStreamSynchronize(g.st));
        std::vector<int> again;
        for (int k : todo) {
            if (!h_sinfo[k]) {
                ok[k] = 1;
                alpha[k] = a[k];
                continue;
            }
            if (++tries[k] >= 40) continue;   // ok[k] stays 0
            a[k] *= 0.8;
            again.push_back(k);
        }
        todo.swap(again);
    }
}

// The least-squares start (solver.c:13939-14198), factored form, per instance
void Lockstep::least_squares_start(std::vector<double> &y, std::vector<char> &started) {
    started.assign(B, 0);
    CU(cudaMemsetAsync(Mm, 0, sizeof(double) * MT, g.st));
    assemble(all, Icat, Icat);   // Q = P with the off-diagonal doubled: M = A A'
    std::vector<int> failed;
    factor(all, failed);
    std::vector<char> okf(B, 1);
    for (int k : failed) okf[k] = 0;
    std::vector<int> L;
    for (int k = 0; k < B; k++)
        if (okf[k]) L.push_back(k);
    if (L.empty()) return;
    std::vector<double> bv(mT, 0.0), dy, AC, yy;
    for (int k : L)
        for (int i = 0; i < m[k]; i++) bv[coff[k] + i] = Pb[k].b[i];
    pcg(L, bv, dy, 1e-8);
    aop(Ccat, AC);
    pcg(L, AC, yy, 1e-8);
    // X = A'dy, Z = C - A'y: instances without a start keep theirs (coefficient 0 below)
    std::vector<double> dyL(mT, 0.0), yL(mT, 0.0);
    for (int k : L)
        for (long long i = coff[k]; i < coff[k + 1]; i++) { dyL[i] = dy[i]; yL[i] = yy[i]; }
    atop(dyL, 1.0, 0.0, cat.T);
    atop(yL, -1.0, 0.0, cat.W);
    std::vector<double> cL(B, 0.0);
    for (int k : L) cL[k] = 1.0;
    set_coef(0, cL);
    {
        std::vector<int> flag(B, 0);
        for (int k : L) flag[k] = 1;
        CU(cudaMemcpyAsync(d_flag, flag.data(), sizeof(int) * B, cudaMemcpyHostToDevice, g.st));
        RC(ew_copy_masked(g.st, B, d_boff, Ntot2, d_flag, cat.T, cat.X));
        RC(ew_lincomb(g.st, Ntot2, 1.0, cat.W, 1.0, Ccat, 0.0, nullptr, cat.W));
        RC(ew_copy_masked(g.st, B, d_boff, Ntot2, d_flag, cat.W, cat.Z));
        CU(cudaStreamSynchronize(g.st));
    }
    // shifts from the exact smallest eigenvalues
    CU(cudaMemcpyAsync(cat.LiX, Icat, sizeof(double) * Ntot2, cudaMemcpyDeviceToDevice, g.st));
    std::vector<double> lx(B), lz(B);
    for (int pass = 0; pass < 2; pass++) {
        RC(small_lammin(g.st, B, d_n, (const double *const *)tab(&DevArrays::LiX),
                        (const double *const *)tab(pass == 0 ? &DevArrays::X : &DevArrays::Z), d_slam));
        CU(cudaMemcpyAsync(h_slam, d_slam, sizeof(double) * B, cudaMemcpyDeviceToHost, g.st));
        CU(cudaStreamSynchronize(g.st));
        for (int k = 0; k < B; k++) (pass == 0 ? lx : lz)[k] = h_slam[k];
    }
    std::vector<double> shx(B, 0.0), shz(B, 0.0);
    for (int k : L) {
        const double ax = -lx[k], az = -lz[k];
        shx[k] = ax >= -1e-8 ? 1.0 + ax : 0.0;
        shz[k] = std::max(0.0, 1.0 + az);
    }
    set_coef(1, shx);
    RC(ew_lincomb_coef(g.st, B, d_boff, Ntot2, d_coef[0], cat.X, d_coef[1], Icat, nullptr, nullptr, cat.T));
    RC(ew_copy_masked(g.st, B, d_boff, Ntot2, d_flag, cat.T, cat.X));
    set_coef(1, shz);
    RC(ew_lincomb_coef(g.st, B, d_boff, Ntot2, d_coef[0], cat.Z, d_coef[1], Icat, nullptr, nullptr, cat.T));
    RC(ew_copy_masked(g.st, B, d_boff, Ntot2, d_flag, cat.T, cat.Z));
    // Cholesky tests, raised where they fail
    for (int pass = 0; pass < 2; pass++) {
        double *DevArrays::*V = pass == 0 ? &DevArrays::X : &DevArrays::Z;
        double *DevArrays::*Lv = pass == 0 ? &DevArrays::LX : &DevArrays::LZ;
        double *DevArrays::*Li = pass == 0 ? &DevArrays::LiX : &DevArrays::LiZ;
        std::vector<double> extra(B, 1e-8);
        for (int round = 0;; round++) {
            RC(small_chol_inv(g.st, B, d_n, tab(V), tab(Lv), tab(Li), d_sinfo));
            CU(cudaMemcpyAsync(h_sinfo, d_sinfo, sizeof(int) * B, cudaMemcpyDeviceToHost, g.st));
            CU(cudaStreamSynchronize(g.st));
            std::vector<double> add(B, 0.0);
            bool any = false;
            for (int k : L)
                if (h_sinfo[k]) {
                    any = true;
                    add[k] = extra[k];
                    extra[k] *= 10;
                    if (extra[k] > 1e31) throw GpuFail{BGPU_ERR_NOTPD, __LINE__};
                }
            if (!any) break;
            set_coef(1, add);
            RC(ew_lincomb_coef(g.st, B, d_boff, Ntot2, d_coef[0], cat.*V, d_coef[1], Icat, nullptr, nullptr, cat.T));
            RC(ew_copy_masked(g.st, B, d_boff, Ntot2, d_flag, cat.T, cat.*V));
        }
    }
    for (int k : L) {
        std::copy(yy.begin() + coff[k], yy.begin() + coff[k + 1], y.begin() + coff[k]);
        started[k] = 1;
    }
    // the factor state starts afresh for the loop
    std::fill(reg.begin(), reg.end(), 0.0);
    std::fill(reg_ok.begin(), reg_ok.end(), 0.0);
    std::fill(reg_hint.begin(), reg_hint.end(), 0);
    std::fill(nfactor.begin(), nfactor.end(), 0);
}

// the DIMACS errors of the returned points on the data as given (as Solver::final_measures)
void Lockstep::final_measures(const std::vector<double> &y, std::vector<ResultData> &res) {
    std::vector<double> cs(B), bs(B);
    for (int k = 0; k < B; k++) { cs[k] = Pb[k].cs; bs[k] = Pb[k].bs; }
    atop(y, -1.0, 0.0, cat.W);   // W = cs (C' - A'(y)), G = bs X
    set_coef(0, cs);
    RC(ew_lincomb_coef(g.st, B, d_boff, Ntot2, d_coef[0], cat.W, d_coef[0], Ccat, nullptr, nullptr, cat.W));
    set_coef(1, bs);
    RC(ew_lincomb_coef(g.st, B, d_boff, Ntot2, d_coef[1], cat.X, nullptr, nullptr, nullptr, nullptr, cat.G));
    std::vector<double> dd;
    {
        const double *aa[2] = {Ccat, cat.G}, *bb[2] = {cat.G, cat.W};
        segdots(2, aa, bb, dd);
    }
    std::vector<double> Xh(Ntot2), Zh(Ntot2);
    CU(cudaMemcpyAsync(Xh.data(), cat.G, sizeof(double) * Ntot2, cudaMemcpyDeviceToHost, g.st));
    CU(cudaMemcpyAsync(Zh.data(), cat.W, sizeof(double) * Ntot2, cudaMemcpyDeviceToHost, g.st));
    CU(cudaMemcpyAsync(cat.LiX, Icat, sizeof(double) * Ntot2, cudaMemcpyDeviceToDevice, g.st));
    std::vector<double> lamz(B, 0.0), lamx(B, 0.0);
    for (int pass = 0; pass < 2; pass++) {
        double *DevArrays::*V = pass == 0 ? &DevArrays::W : &DevArrays::G;
        RC(small_chol_inv(g.st, B, d_n, tab(V), tab(&DevArrays::T), nullptr, d_sinfo));
        RC(small_lammin(g.st, B, d_n, (const double *const *)tab(&DevArrays::LiX), (const double *const *)tab(V), d_slam));
        CU(cudaMemcpyAsync(h_sinfo, d_sinfo, sizeof(int) * B, cudaMemcpyDeviceToHost, g.st));
        CU(cudaMemcpyAsync(h_slam, d_slam, sizeof(double) * B, cudaMemcpyDeviceToHost, g.st));
        CU(cudaStreamSynchronize(g.st));
        for (int k = 0; k < B; k++)
            if (h_sinfo[k]) (pass == 0 ? lamz : lamx)[k] = std::max(0.0, -h_slam[k]);
    }
    std::vector<double> AX;
    aop(cat.G, AX);
    for (int k = 0; k < B; k++) {
        ResultData &r = res[k];
        const HProblem &P = Pb[k];
        const long long nn = (long long)n[k] * n[k];
        r.y.resize(m[k]);
        for (int i = 0; i < m[k]; i++) r.y[i] = cs[k] * P.d[i] * y[coff[k] + i];
        r.X.assign(1, std::vector<double>(Xh.begin() + boff[k], Xh.begin() + boff[k] + nn));
        r.Z.assign(1, std::vector<double>(Zh.begin() + boff[k], Zh.begin() + boff[k] + nn));
        const double pobj = cs[k] * dd[(size_t)k * 2 + 0], xz = dd[(size_t)k * 2 + 1];
        double r2 = 0, dobj = 0;
        for (int i = 0; i < m[k]; i++) {
            const double v = AX[coff[k] + i] / P.d[i] - P.b0[i];
            r2 += v * v;
            dobj += P.b0[i] * r.y[i];
        }
        const double den = 1 + std::fabs(pobj) + std::fabs(dobj);
        r.err[1] = std::sqrt(r2) / (1 + P.normb1);
        r.err[2] = lamx[k] / (1 + P.normb1);
        r.err[3] = 0;
        r.err[4] = lamz[k] / (1 + P.normC1);
        r.err[5] = (pobj - dobj) / den;
        r.err[6] = xz / den;
        r.pobj = pobj;
        r.dobj = dobj;
        r.have_x = 1;
        r.d2h_bytes = 2.0 * sizeof(double) * (double)nn;
    }
}

void Lockstep::run(std::vector<ResultData> &res) {
    const double t0 = wtime();
    res.assign(B, ResultData());
    std::fill(pcg_iters.begin(), pcg_iters.end(), 0);
    std::fill(nfactor.begin(), nfactor.end(), 0);
    std::fill(reg.begin(), reg.end(), 0.0);
    std::fill(reg_ok.begin(), reg_ok.end(), 0.0);
    std::fill(reg_hint.begin(), reg_hint.end(), 0);
    schur_flops = 0;
    t_start = t_asm = t_fac = t_pcg = t_loop = t_final = 0;
    CU(cudaEventRecord(ev0, g.st));
    std::vector<double> y(mT, 0.0), ybest(mT, 0.0), dy, rp(mT), a0, h(mT, 0.0), rhs(mT), qv, ev(mT), wv;
    // start_sdpt3 (solver.c:6622-6661): X = xi I, Z = eta I and their factors, closed form
    {
        std::vector<std::vector<double>> sv(6, std::vector<double>(B, 0.0));
        for (int k = 0; k < B; k++) {
            const double xi = Pb[k].xi0, eta = Pb[k].eta0;
            sv[0][k] = xi;
            sv[1][k] = eta;
            sv[2][k] = std::sqrt(xi);
            sv[3][k] = std::sqrt(eta);
            sv[4][k] = 1.0 / std::sqrt(xi);
            sv[5][k] = 1.0 / std::sqrt(eta);
        }
        double *DevArrays::*mems[6] = {&DevArrays::X, &DevArrays::Z, &DevArrays::LX, &DevArrays::LZ, &DevArrays::LiX,
                                       &DevArrays::LiZ};
        for (int q = 0; q < 6; q++) {
            set_coef(0, sv[q]);
            RC(ew_scaled_identity_blocks(g.st, B, d_n, d_boff, Ntot2, d_coef[0], nullptr, cat.*mems[q]));
        }
        CU(cudaStreamSynchronize(g.st));
    }
    std::vector<char> started;
    if (opt.init >= 1) least_squares_start(y, started);
    t_start = wtime() - t0;
    const double t_a0 = t_asm, t_f0 = t_fac, t_p0 = t_pcg;
    // R0 = C - Z - A'y, theta = 1
    std::vector<double> theta(B, 1.0), r0norm(B, 0.0);
    atop(y, -1.0, 0.0, cat.R0);
    RC(ew_lincomb(g.st, Ntot2, 1.0, Ccat, -1.0, cat.Z, 1.0, cat.R0, cat.R0));
    {
        std::vector<double> dd;
        const double *aa[1] = {cat.R0};
        segdots(1, aa, aa, dd);
        for (int k = 0; k < B; k++) r0norm[k] = std::sqrt(dd[k]);
    }
    std::vector<double> nbs(B, 0.0);
    for (int k = 0; k < B; k++) {
        double s = 0;
        for (double v : Pb[k].b) s += v * v;
        nbs[k] = std::sqrt(s);
    }
    std::vector<int> status(B, -1), it_best(B, 0), stall(B, 0), iters(B, 0);
    std::vector<double> alp(B, 0.0), ald(B, 0.0), sigma(B, 0.0), best_score(B, INFINITY), mu(B, 0.0);
    std::vector<IterRes> R(B), best(B);
    std::vector<double> ones(B, 1.0), zeros(B, 0.0), coefv(B, 0.0);
    int it = 0;
    for (it = 0; it <= opt.maxit; it++) {
        std::vector<int> act;
        for (int k = 0; k < B; k++)
            if (status[k] < 0) act.push_back(k);
        if (act.empty()) break;
        if (nt) {   // the NT scaling (solver.c:7898-7912): G, lam and W = G G' (in Zi); a failure ends the instance
            RC(nt::scaling_small(g.st, B, d_n, nmax, (const double *const *)tab(&DevArrays::LX),
                                 (const double *const *)tab(&DevArrays::LZ), tab(&DevArrays::NG), d_lamtab,
                                 tab(&DevArrays::Zi), d_ntinfo));
            CU(cudaMemcpyAsync(h_ntinfo, d_ntinfo, sizeof(int) * B, cudaMemcpyDeviceToHost, g.st));
            CU(cudaStreamSynchronize(g.st));
            std::vector<int> keep;
            for (int k : act) {
                if (h_ntinfo[k]) status[k] = 4;
                else keep.push_back(k);
            }
            act.swap(keep);
            if (act.empty()) break;
        } else {   // Zi = LiZ' LiZ
            RC(small_gemm(g.st, B, d_n, 1, 0, 1.0, (const double *const *)tab(&DevArrays::LiZ),
                          (const double *const *)tab(&DevArrays::LiZ), 0.0, tab(&DevArrays::Zi), 1));
        }
        double *DevArrays::*Xw = nt ? &DevArrays::Zi : &DevArrays::X;   // X, or W under NT (nt_view)
        // residuals and objectives
        std::vector<double> AX;
        aop(cat.X, AX);
        for (int k : act)
            for (int i = 0; i < m[k]; i++) rp[coff[k] + i] = Pb[k].b[i] - AX[coff[k] + i];
        atop(y, 1.0, 0.0, cat.F);
        RC(ew_lincomb(g.st, Ntot2, 1.0, cat.F, 1.0, cat.Z, 0.0, nullptr, cat.F));
        RC(ew_lincomb(g.st, Ntot2, 1.0, cat.F, -1.0, Ccat, 0.0, nullptr, cat.Fd));
        set_coef(0, ones);
        set_coef(1, theta);
        RC(ew_lincomb_coef(g.st, B, d_boff, Ntot2, d_coef[0], cat.Fd, d_coef[1], cat.R0, nullptr, nullptr, cat.T));
        std::vector<double> part;
        {
            const double *aa[5] = {cat.F, Ccat, cat.X, cat.Fd, cat.T}, *bb[5] = {cat.F, cat.X, cat.Z, cat.Fd, cat.T};
            segdots(5, aa, bb, part);
        }
        std::vector<int> flag_best(B, 0), flag_rebase(B, 0);
        std::vector<double> xz(B, 0.0);
        for (int k : act) {
            const HProblem &P = Pb[k];
            const double nCR2 = part[k * 5 + 0], pobj = part[k * 5 + 1], xzk = part[k * 5 + 2], rdn2 = part[k * 5 + 3],
                         dev2 = part[k * 5 + 4];
            xz[k] = xzk;
            double dobj = 0;
            for (int i = 0; i < m[k]; i++) dobj += P.b[i] * y[coff[k] + i];
            mu[k] = xzk / (double)P.Ntot;
            double rpo = 0;
            for (int i = 0; i < m[k]; i++) { const double v = rp[coff[k] + i] * P.du[i]; rpo += v * v; }
            rpo = std::sqrt(rpo);
            const double rdo = P.cs * std::sqrt(rdn2);
            const double sc = P.bs * P.cs;
            const double po = sc * pobj, dob = sc * dobj;
            IterRes &Rk = R[k];
            Rk.pobj = po;
            Rk.dobj = dob;
            Rk.pinf = rpo / (1 + P.normb2);
            Rk.dinf = rdo / (1 + P.normC2);
            const double oden = 1 + std::fabs(po) + std::fabs(dob);
            Rk.relgap = std::fabs(po - dob) / oden;
            Rk.relcomp = sc * xzk / oden;
            Rk.err[1] = rpo / (1 + P.normb1);
            Rk.err[3] = rdo / (1 + P.normC1);
            Rk.err[5] = (po - dob) / oden;
            Rk.err[6] = sc * xzk / oden;
            iters[k] = it;
            if (!std::isfinite(po) || !std::isfinite(dob)) { status[k] = 4; continue; }
            const double score = res_score(Rk);
            if (score < best_score[k]) {
                best_score[k] = score;
                it_best[k] = it;
                best[k] = Rk;
                std::copy(y.begin() + coff[k], y.begin() + coff[k + 1], ybest.begin() + coff[k]);
                flag_best[k] = 1;
            }
            if (score < opt.tol) { status[k] = 0; continue; }
            if (it > it_best[k] && dimacs_score(best[k]) <= 0.5 * opt.tol) { status[k] = 4; continue; }
            if (opt.timelimit > 0 && wtime() - t0 > opt.timelimit) { status[k] = 6; continue; }
            const double nCR = std::sqrt(nCR2);
            if (!opt.known_feasible && dobj > 0 && nCR / dobj < 1e-8 && it > 5) { status[k] = 1; continue; }
            double nAX = 0;
            for (int i = 0; i < m[k]; i++) { const double v = P.b[i] - rp[coff[k] + i]; nAX += v * v; }
            nAX = std::sqrt(nAX);
            if (!opt.known_feasible && pobj < 0 && nAX / (-pobj) < 1e-8 && it > 5) { status[k] = 2; continue; }
            if (it == opt.maxit) { status[k] = 3; continue; }
            if (stall[k] >= 3) { status[k] = 4; continue; }
            if (it - it_best[k] >= opt.stall_win && best_score[k] < 1e-6) { status[k] = 4; continue; }
            if (it - it_best[k] >= 8 && best_score[k] < 1e-4) { status[k] = 4; continue; }
            if (it - it_best[k] >= 12) { status[k] = 4; continue; }
            const double dev = std::sqrt(dev2);
            if (dev > 1e-10 * (1.0 + theta[k] * r0norm[k]) && dev > 1e-12) {
                theta[k] = 1.0;
                r0norm[k] = std::sqrt(rdn2);
                flag_rebase[k] = 1;
            }
            if (theta[k] * r0norm[k] <= 1e-13) theta[k] = 0.0;
        }
        {   // the best iterate's X and Z; the re-based R0 = -Fd
            CU(cudaMemcpyAsync(d_flag, flag_best.data(), sizeof(int) * B, cudaMemcpyHostToDevice, g.st));
            RC(ew_copy_masked(g.st, B, d_boff, Ntot2, d_flag, cat.X, cat.Xb));
            RC(ew_copy_masked(g.st, B, d_boff, Ntot2, d_flag, cat.Z, cat.Zb));
            CU(cudaStreamSynchronize(g.st));
            RC(ew_lincomb(g.st, Ntot2, -1.0, cat.Fd, 0.0, nullptr, 0.0, nullptr, cat.Bm));
            CU(cudaMemcpyAsync(d_flag, flag_rebase.data(), sizeof(int) * B, cudaMemcpyHostToDevice, g.st));
            RC(ew_copy_masked(g.st, B, d_boff, Ntot2, d_flag, cat.Bm, cat.R0));
            CU(cudaStreamSynchronize(g.st));
        }
        act.clear();
        for (int k = 0; k < B; k++)
            if (status[k] < 0) act.push_back(k);
        if (act.empty()) break;
        // ---- Schur complement and its factor ----
        assemble(act, cat.*Xw, cat.Zi);
        std::vector<int> failed;
        factor(act, failed);
        for (int k : failed) status[k] = 4;
        if (!failed.empty()) {
            act.clear();
            for (int k = 0; k < B; k++)
                if (status[k] < 0) act.push_back(k);
            if (act.empty()) break;
        }
        std::vector<double> dmask(B, 0.0);   // 1 on the active instances
        for (int k : act) dmask[k] = 1.0;
        // ---- rhs pieces: a0 = A(Zi) (HKM), h = A(theta Zi R0 X) (W theta R0 W under NT) ----
        if (!nt) aop(cat.Zi, a0);
        mul(&DevArrays::Zi, &DevArrays::R0, &DevArrays::T);
        set_coef(1, theta);
        RC(ew_lincomb_coef(g.st, B, d_boff, Ntot2, d_coef[1], cat.T, nullptr, nullptr, nullptr, nullptr, cat.T));
        mul(&DevArrays::T, Xw, &DevArrays::G);
        aop(cat.G, h);
        // ---- predictor ----
        for (int k : act)
            for (int i = 0; i < m[k]; i++) rhs[coff[k] + i] = Pb[k].b[i] + h[coff[k] + i];
        pcg(act, rhs, dy, 1e-7);
        atop(dy, -1.0, 0.0, cat.dZ);
        set_coef(0, ones);
        set_coef(1, theta);
        RC(ew_lincomb_coef(g.st, B, d_boff, Ntot2, d_coef[0], cat.dZ, d_coef[1], cat.R0, nullptr, nullptr, cat.dZ));
        if (nt) {   // scaled: dXt = Rt - G' dZ G with Rt = -diag(lam), dX = G dXt G' (solver.c:14740-14792)
            RC(nt::rhs_scaled(g.st, B, d_n, d_boff, d_loff, Ntot2, nlam, 0.0, nullptr, cat.Rt));
            nt_toZ(&DevArrays::dZ, &DevArrays::dZt);
            RC(ew_lincomb(g.st, Ntot2, 1.0, cat.Rt, -1.0, cat.dZt, 0.0, nullptr, cat.dXt));
            nt_fromS(&DevArrays::dXt, &DevArrays::dX);
        } else {
            mul(&DevArrays::Zi, &DevArrays::dZ, &DevArrays::T);
            mul(&DevArrays::T, &DevArrays::X, &DevArrays::G);
            RC(ew_sym_lincomb_blocks(g.st, B, d_n, d_boff, Ntot2, cat.G, -1.0, -1.0, cat.X, 0.0, nullptr, cat.dX));
        }
        std::vector<double> ap, ad;
        maxstep(1, ap);
        maxstep(0, ad);
        std::vector<double> t3;
        {
            const double *aa[3] = {cat.X, cat.dX, cat.dX}, *bb[3] = {cat.dZ, cat.Z, cat.dZ};
            segdots(3, aa, bb, t3);
        }
        std::vector<double> gamma(B, 0.9), smu(B, 0.0);
        for (int k : act) {
            ap[k] = std::min(1.0, ap[k]);
            ad[k] = std::min(1.0, ad[k]);
            const double xdz = t3[k * 3 + 0], dxz = t3[k * 3 + 1], dxdz = t3[k * 3 + 2];
            const double Ntot = (double)Pb[k].Ntot;
            const double mu_a = (xz[k] + ap[k] * dxz + ad[k] * xdz + ap[k] * ad[k] * dxdz) / Ntot;
            const double frac = std::max(0.0, mu_a / mu[k]);
            const double mina = std::min(ap[k], ad[k]);
            const int rule = opt.sigma_rule < 0 ? 0 : opt.sigma_rule;
            double expon;
            if (rule == 1) expon = 3.0;
            else if (rule == 2) expon = (mina < 0.1) ? 1.0 : 3.0;
            else expon = (R[k].relgap > 1e-6) ? std::max(1.0, 3 * mina * mina) : 3.0;
            double sg = std::min(1.0, std::pow(frac, expon));
            if (sg < opt.sigma_min) sg = opt.sigma_min;
            const double infeas = std::max(R[k].pinf, R[k].dinf), bal = opt.balance;
            if (bal > 0 && infeas > bal * R[k].relcomp && R[k].relcomp > 0) {
                const double s_min = std::min(1.0, infeas / (bal * R[k].relcomp) * 0.1);
                if (sg < s_min) sg = s_min;
            }
            sigma[k] = sg;
            gamma[k] = 0.9 + (opt.gamma_max - 0.9) * mina;
            smu[k] = sg * mu[k];
        }
        // ---- corrector ----
        if (nt) {   // Rt = L_lam^-1(smu I - lam^2 - sym(dXt dZt)), rhs = b + h - A(G (Rt + lam) G') (solver.c:14876-14906)
            RC(small_gemm(g.st, B, d_n, 0, 0, 1.0, (const double *const *)tab(&DevArrays::dXt),
                          (const double *const *)tab(&DevArrays::dZt), 0.0, tab(&DevArrays::W), 1));
            set_coef(3, smu);
            RC(nt::rhs_scaled(g.st, B, d_n, d_boff, d_loff, Ntot2, nlam, 0.0, cat.W, cat.Rt, d_coef[3]));
            RC(nt::add_lam(g.st, B, d_n, d_boff, d_loff, Ntot2, nlam, 1.0, cat.Rt, cat.Q));
            nt_fromS(&DevArrays::Q, &DevArrays::G);
            aop(cat.G, qv);
            for (int k : act)
                for (int i = 0; i < m[k]; i++) {
                    const long long c = coff[k] + i;
                    rhs[c] = Pb[k].b[i] + h[c] - qv[c];
                }
        } else {
            mul(&DevArrays::Zi, &DevArrays::dZ, &DevArrays::T);
            mul(&DevArrays::T, &DevArrays::dX, &DevArrays::Q);   // Q = Zi dZp dXp
            aop(cat.Q, qv);
            for (int k : act)
                for (int i = 0; i < m[k]; i++) {
                    const long long c = coff[k] + i;
                    rhs[c] = Pb[k].b[i] - smu[k] * a0[c] + qv[c] + h[c];
                }
        }
        pcg(act, rhs, dy, 0);
        atop(dy, -1.0, 0.0, cat.dZ);
        set_coef(0, ones);
        set_coef(1, theta);
        RC(ew_lincomb_coef(g.st, B, d_boff, Ntot2, d_coef[0], cat.dZ, d_coef[1], cat.R0, nullptr, nullptr, cat.dZ));
        if (nt) {   // dX = G (Rt - G' dZ G) G' (solver.c:14976-14996)
            nt_toZ(&DevArrays::dZ, &DevArrays::Q);
            RC(ew_lincomb(g.st, Ntot2, 1.0, cat.Rt, -1.0, cat.Q, 0.0, nullptr, cat.W));
            nt_fromS(&DevArrays::W, &DevArrays::dX);
        } else {
            mul(&DevArrays::Zi, &DevArrays::dZ, &DevArrays::T);
            mul(&DevArrays::T, &DevArrays::X, &DevArrays::G);
            RC(ew_lincomb(g.st, Ntot2, 1.0, cat.G, 1.0, cat.Q, 0.0, nullptr, cat.G));   // Zi dZ X + Q
            std::vector<double> mones(B, -1.0);
            set_coef(0, mones);
            set_coef(1, smu);
            set_coef(2, mones);
            RC(ew_sym_coef(g.st, B, d_n, d_boff, Ntot2, cat.G, d_coef[0], d_coef[1], cat.Zi, d_coef[2], cat.X, cat.dX));
        }
        // ---- refinement of A(dX) = rp, per instance ----
        {
            std::vector<int> ref = act;
            for (int pass = 0; pass < 3 && !ref.empty(); pass++) {
                std::vector<double> AdX;
                aop(cat.dX, AdX);
                std::vector<int> go;
                std::vector<double> ne(B, 0.0);
                std::fill(ev.begin(), ev.end(), 0.0);
                for (int k : ref) {
                    double s1 = 0, s2 = 0;
                    for (long long c = coff[k]; c < coff[k + 1]; c++) {
                        ev[c] = rp[c] - AdX[c];
                        s1 += ev[c] * ev[c];
                        s2 += rp[c] * rp[c];
                    }
                    ne[k] = std::sqrt(s1);
                    const double nrp = std::sqrt(s2);
                    if (ne[k] > 1e-2 * nrp && ne[k] > 1e-3 * opt.tol * (1 + nbs[k])) go.push_back(k);
                }
                if (go.empty()) break;
                pcg(go, ev, wv, 0);
                atop(wv, 1.0, 0.0, cat.W);   // A'w (zero on the instances outside go)
                mul(&DevArrays::Zi, &DevArrays::W, &DevArrays::T);
                mul(&DevArrays::T, Xw, &DevArrays::F);   // Zi A'w X (W A'w W under NT)
                RC(ew_sym_lincomb_blocks(g.st, B, d_n, d_boff, Ntot2, cat.F, 1.0, 0.0, nullptr, 0.0, nullptr, cat.G));
                std::vector<double> AG;
                aop(cat.G, AG);
                std::vector<int> keep;
                std::vector<double> cw(B, 0.0), cg(B, 0.0);
                for (int k : go) {
                    double s = 0;
                    for (long long c = coff[k]; c < coff[k + 1]; c++) { const double v = ev[c] - AG[c]; s += v * v; }
                    if (!(std::sqrt(s) < 0.5 * ne[k])) continue;
                    for (long long c = coff[k]; c < coff[k + 1]; c++) dy[c] += wv[c];
                    cw[k] = -1.0;
                    cg[k] = 1.0;
                    keep.push_back(k);
                }
                if (!keep.empty()) {
                    set_coef(0, ones);
                    set_coef(1, cw);
                    RC(ew_lincomb_coef(g.st, B, d_boff, Ntot2, d_coef[0], cat.dZ, d_coef[1], cat.W, nullptr, nullptr,
                                       cat.dZ));
                    set_coef(1, cg);
                    RC(ew_lincomb_coef(g.st, B, d_boff, Ntot2, d_coef[0], cat.dX, d_coef[1], cat.G, nullptr, nullptr,
                                       cat.dX));
                }
                ref.swap(keep);
            }
        }
        std::vector<double> apr, adr;
        maxstep(1, apr);
        maxstep(0, adr);
        std::vector<double> apn(B, 0.0), adn(B, 0.0);
        for (int k : act) {
            apn[k] = std::min(1.0, gamma[k] * std::min(1.0, apr[k]));
            adn[k] = std::min(1.0, gamma[k] * std::min(1.0, adr[k]));
        }
        // catastrophe guard (solver.c:15138-15158)
        {
            bool any = false;
            for (int k : act) any = any || R[k].pinf < 1e-6;
            if (any) {
                std::vector<double> AdX;
                aop(cat.dX, AdX);
                for (int k : act) {
                    if (!(R[k].pinf < 1e-6)) continue;
                    double s1 = 0, s2 = 0;
                    for (long long c = coff[k]; c < coff[k + 1]; c++) {
                        const double v = rp[c] - AdX[c];
                        s1 += v * v;
                        s2 += rp[c] * rp[c];
                    }
                    const double nrp = std::sqrt(s2), nev = std::sqrt(s1);
                    const double gg = std::max(1e3, 1e-6 / std::max(R[k].pinf, 1e-300));
                    const double lim = gg * nrp;
                    if (nev > lim && nrp > 0) apn[k] = std::min(apn[k], lim / nev);
                }
            }
        }
        std::vector<char> okp, okd;
        try_step(1, act, apn, okp);
        try_step(0, act, adn, okd);
        for (int k : act) {
            if (!okp[k] || !okd[k]) { status[k] = 4; continue; }
            for (long long c = coff[k]; c < coff[k + 1]; c++) y[c] += adn[k] * dy[c];
            theta[k] *= (1.0 - adn[k]);
            alp[k] = apn[k];
            ald[k] = adn[k];
            stall[k] = (apn[k] < 1e-6 && adn[k] < 1e-6) ? stall[k] + 1 : 0;
        }
    }
    // fall back to the best iterate seen
    {
        std::vector<int> flag(B, 0);
        for (int k = 0; k < B; k++) {
            if (status[k] < 0) status[k] = 3;
            if (status[k] != 0 && status[k] != 1 && status[k] != 2 && best_score[k] < res_score(R[k])) {
                R[k] = best[k];
                std::copy(ybest.begin() + coff[k], ybest.begin() + coff[k + 1], y.begin() + coff[k]);
                flag[k] = 1;
            }
        }
        CU(cudaMemcpyAsync(d_flag, flag.data(), sizeof(int) * B, cudaMemcpyHostToDevice, g.st));
        RC(ew_copy_masked(g.st, B, d_boff, Ntot2, d_flag, cat.Xb, cat.X));
        RC(ew_copy_masked(g.st, B, d_boff, Ntot2, d_flag, cat.Zb, cat.Z));
        CU(cudaStreamSynchronize(g.st));
    }
    const double tl = wtime();
    t_loop = tl - t0 - t_start - (t_asm - t_a0) - (t_fac - t_f0) - (t_pcg - t_p0);
    final_measures(y, res);
    t_final = wtime() - tl;
    const double tt = wtime() - t0;
    CU(cudaEventRecord(ev1, g.st));
    CU(cudaEventSynchronize(ev1));
    float dms = 0;
    CU(cudaEventElapsedTime(&dms, ev0, ev1));
    for (int k = 0; k < B; k++) {
        ResultData &r = res[k];
        int st = status[k];
        const double acc = std::max(std::max(r.err[1], r.err[2]),
                                    std::max(r.err[4], std::max(std::fabs(r.err[5]), std::fabs(r.err[6]))));
        if (st == 0 || st == 5 || st == 3 || st == 4 || st == 6) {
            if (acc <= opt.tol) st = 0;
            else if (acc <= opt.red_acc) st = 5;
            else if (st == 0 || st == 5) st = 4;
        }
        r.status = st;
        r.exit_code = exit_code_of(st);
        r.iters = iters[k];
        r.m = m[k];
        r.nblk = 1;
        r.bs = {n[k]};
        r.nfactor = nfactor[k];
        r.pcg_iters = pcg_iters[k];
        r.time = tt;
        r.device_time = dms * 1e-3;   // CUDA events on the batch's stream around the whole solve
        r.schur_flops = schur_flops / B;
    }
}
