/*
 * orc_sampler.c -- oracle restatement of the reference's samplers,
 * aggregators and SR/CG solver (TEST INFRASTRUCTURE ONLY; see orc.h).
 *
 * Metropolis randomness: the reference draws from std::mt19937, which cannot
 * be reproduced on a GPU bit-for-bit and need not be.  Oracle and CUDA
 * sampler both draw from Philox4x32-10 with the same counter layout, so the
 * two produce identical chains up to floating-point ties in the acceptance
 * test:  counter = {proposal index, epoch, chain, stream}, key = seed.
 *   stream 0: proposals -> (w0: bond-or-site, w1: index, w2: acceptance)
 *   stream 1: initial configuration bits (w0..w3 = sites 0..127)
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "orc.h"

static inline int bit(const uint32_t* s, int i) { return (s[i >> 5] >> (i & 31)) & 1; }
static inline double sig(const uint32_t* s, int i) { return bit(s, i) ? -1.0 : 1.0; }
static inline double unit24(uint32_t x) { return (double)(x >> 8) * (1.0 / 16777216.0); }
static inline uint32_t pick(uint32_t x, uint32_t n) { return (uint32_t)(((uint64_t)x * n) >> 32); }

static void lncosh_terms(const double complex* th, int T, double complex* out) {
    for (int t = 0; t < T; t++) out[t] = orc_lncosh_sum(th + t, 1);
}

/* metropolis_sampler::sample_chain, metropolis_sampler.cpp:118-273.
 * The RBM context (theta) is updated incrementally as in the reference;
 * psi ratios use sum lncosh(theta') - sum lncosh(theta)
 * (rbm_base.cpp:320-344).  The Pfaffian context is updated by the rank-2m
 * update with a refresh every pf_refresh accepted moves
 * (abstract_sampler.cpp:103-113). */
static double run_chain(const orc_machine* m, const orc_ops* ops,
                        const orc_sampler_cfg* cfg, uint32_t epoch, int chain,
                        int init, uint32_t* spins, double complex* E,
                        double complex* O) {
    int n = m->n, nh = m->nh, S = m->S, T = nh * S, P = orc_n_params(m);
    uint32_t key[2] = {(uint32_t)cfg->seed, (uint32_t)(cfg->seed >> 32)};
    if (init) {
        uint32_t ctr[4] = {0, epoch, (uint32_t)chain, 1}, r[4];
        orc_philox(ctr, key, r);
        for (int w = 0; w < 4; w++) {
            int lo = 32 * w;
            uint32_t mask = n >= lo + 32 ? 0xffffffffu : (n > lo ? ((1u << (n - lo)) - 1) : 0);
            spins[w] = r[w] & mask;
        }
    }
    double complex* th = (double complex*)malloc(sizeof(double complex) * T);
    double complex* th2 = (double complex*)malloc(sizeof(double complex) * T);
    orc_theta(m, spins, th);
    double complex lc = orc_lncosh_sum(th, T);
    orc_pfctx pc, pc2;
    pc.inv = pc2.inv = NULL;
    if (m->has_pf) {
        pc.inv = (double complex*)malloc(sizeof(double complex) * n * n);
        pc2.inv = (double complex*)malloc(sizeof(double complex) * n * n);
        orc_pf_context(m, spins, &pc);
    }
    int spc = cfg->samples_per_chain;
    int warm = cfg->warmup;
    long total = (long)spc * cfg->step + warm;
    uint32_t prop = 0;
    long accepted = 0;
    int ar = 0;
    for (long st = 0; st < total; st++) {
        int slot = 0;
        while (slot < n) {
            uint32_t ctr[4] = {prop, epoch, (uint32_t)chain, 0}, r[4];
            orc_philox(ctr, key, r);
            prop++;
            int fl[2], nf;
            if (cfg->n_prop_bonds > 0 && cfg->bond_flips > 0 && unit24(r[0]) < cfg->bond_flips) {
                uint32_t b = pick(r[1], (uint32_t)cfg->n_prop_bonds);
                fl[0] = cfg->prop_bonds[2 * b];
                fl[1] = cfg->prop_bonds[2 * b + 1];
                nf = 2;
                slot += 2;
            } else {
                fl[0] = (int)pick(r[1], (uint32_t)n);
                nf = 1;
                slot += 1;
            }
            /* psi'/psi for the proposal */
            double complex lr = 0;
            for (int q = 0; q < nf; q++) lr -= 2.0 * sig(spins, fl[q]) * m->v[fl[q] % m->n_vb];
            memcpy(th2, th, sizeof(double complex) * T);
            for (int s = 0; s < S; s++)
                for (int q = 0; q < nf; q++) {
                    int f = fl[q];
                    int p = m->perm ? m->perm[s * n + f] : f;
                    double sf = sig(spins, f);
                    for (int k = 0; k < nh; k++) th2[k + nh * s] -= 2.0 * sf * m->W[p + n * k];
                }
            double complex lc2 = orc_lncosh_sum(th2, T);
            lr += lc2 - lc;
            double a2 = exp(2.0 * creal(lr));
            if (m->has_pf) {
                memcpy(pc2.inv, pc.inv, sizeof(double complex) * n * n);
                pc2.pf_mant = pc.pf_mant;
                pc2.pf_exp10 = pc.pf_exp10;
                orc_pf_update(m, spins, fl, nf, &pc2);
                double uf = cabs(pc2.update_factor);
                a2 *= uf * uf;
            }
            if (unit24(r[2]) < a2) {
                double complex* t = th;
                th = th2;
                th2 = t;
                lc = lc2;
                for (int q = 0; q < nf; q++) spins[fl[q] >> 5] ^= 1u << (fl[q] & 31);
                accepted++;
                ar++;
                if (m->has_pf) {
                    if (cfg->pf_refresh && ar % cfg->pf_refresh == 0) {
                        orc_pf_context(m, spins, &pc);
                    } else {
                        double complex* t2 = pc.inv;
                        pc.inv = pc2.inv;
                        pc2.inv = t2;
                        pc.pf_mant = pc2.pf_mant;
                        pc.pf_exp10 = pc2.pf_exp10;
                    }
                }
            }
        }
        if (st >= warm && (st - warm) % cfg->step == 0) {
            long j = (st - warm) / cfg->step;
            size_t idx = (size_t)chain * spc + j;
            if (E) E[idx] = orc_eloc(m, ops, spins);
            if (O) orc_derivative(m, spins, O + idx * P);
        }
    }
    free(th);
    free(th2);
    free(pc.inv);
    free(pc2.inv);
    (void)lncosh_terms;
    return prop ? (double)accepted / (double)prop : 0.0;
}

void orc_metropolis(const orc_machine* m, const orc_ops* ops,
                    const orc_sampler_cfg* cfg, uint32_t epoch, int init,
                    uint32_t* spins_io, double complex* E, double complex* O,
                    double* acc_chain, int n_threads) {
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < cfg->n_chains; c++) {
        double a = run_chain(m, ops, cfg, epoch, c, init, spins_io + 4 * c, E, O);
        if (acc_chain) acc_chain[c] = a;
    }
}

/* full_sampler::sample, full_sampler.cpp:43-186: all 2^n configurations
 * weighted by p = |psi|^2 (normalised by the largest |psi|^2 here, which
 * cancels in every ratio the aggregators form). */
void orc_full(const orc_machine* m, const orc_ops* ops, double* p_tot,
              double complex* E_mean, double complex* d, double complex* dh,
              double* var_O, int n_threads) {
    int n = m->n, P = orc_n_params(m);
    long NS = 1L << n;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
    double* lp = (double*)malloc(sizeof(double) * NS);
    double mx = -1e300;
#pragma omp parallel for reduction(max : mx)
    for (long x = 0; x < NS; x++) {
        uint32_t s[4] = {(uint32_t)x, (uint32_t)(x >> 32), 0, 0};
        lp[x] = 2.0 * creal(orc_log_psi(m, s));
        if (lp[x] > mx) mx = lp[x];
    }
    double pt = 0;
    double complex em = 0;
    double complex* dd = (double complex*)calloc(P, sizeof(double complex));
    double complex* ddh = (double complex*)calloc(P, sizeof(double complex));
    double* d2 = (double*)calloc(P, sizeof(double));
#pragma omp parallel
    {
        double complex* O = (double complex*)malloc(sizeof(double complex) * P);
        double complex* ld = (double complex*)calloc(P, sizeof(double complex));
        double complex* ldh = (double complex*)calloc(P, sizeof(double complex));
        double* l2 = (double*)calloc(P, sizeof(double));
        double lpt = 0;
        double complex lem = 0;
#pragma omp for schedule(static)
        for (long x = 0; x < NS; x++) {
            uint32_t s[4] = {(uint32_t)x, (uint32_t)(x >> 32), 0, 0};
            double p = exp(lp[x] - mx);
            double complex e = orc_eloc(m, ops, s);
            lpt += p;
            lem += p * e;
            if (d) {
                orc_derivative(m, s, O);
                for (int k = 0; k < P; k++) {
                    ld[k] += p * O[k];
                    ldh[k] += p * e * conj(O[k]);
                    l2[k] += p * (creal(O[k]) * creal(O[k]) + cimag(O[k]) * cimag(O[k]));
                }
            }
        }
#pragma omp critical
        {
            pt += lpt;
            em += lem;
            for (int k = 0; k < P; k++) {
                dd[k] += ld[k];
                ddh[k] += ldh[k];
                d2[k] += l2[k];
            }
        }
        free(O);
        free(ld);
        free(ldh);
        free(l2);
    }
    *p_tot = pt;
    *E_mean = em / pt;
    if (d) {
        for (int k = 0; k < P; k++) {
            d[k] = dd[k] / pt;
            dh[k] = ddh[k] / pt;
            if (var_O) {
                double m2 = d2[k] / pt - (creal(d[k]) * creal(d[k]) + cimag(d[k]) * cimag(d[k]));
                var_O[k] = m2 < 0 ? 0 : m2;
            }
        }
    }
    free(lp);
    free(dd);
    free(ddh);
    free(d2);
}

/* ------------------------------------------------------------- stats --- */
/* aggregator::aggregate + finalize for unit weights (aggregator.cpp:84-239):
 * mean, M2 = sum |x - mean|^2, bin means over consecutive samples,
 * tau = 0.5 (max(bin_size * M2_bin / M2, 1) - 1), variances divided by N-1,
 * stddev = sqrt(var_binned / n_bins) (or sqrt(var / N) without bins). */
void orc_stats(const double complex* x, int N, int n_bins, double complex* mean,
               double* var, double* var_binned, double* tau, double* stddev) {
    double complex mu = 0;
    for (int i = 0; i < N; i++) mu += x[i];
    mu /= N;
    double m2 = 0;
    for (int i = 0; i < N; i++) {
        double complex d = x[i] - mu;
        m2 += creal(d) * creal(d) + cimag(d) * cimag(d);
    }
    double m2b = 0;
    int binning = n_bins > 1;
    if (binning) {
        int bs = N / n_bins;
        for (int b = 0; b < n_bins; b++) {
            double complex bm = 0;
            for (int i = 0; i < bs; i++) bm += x[b * bs + i];
            bm /= bs;
            double complex d = bm - mu;
            m2b += bs * (creal(d) * creal(d) + cimag(d) * cimag(d));
        }
        double t;
        if (m2 == 0 && m2b == 0)
            t = 0;
        else {
            double r = bs * m2b / m2;
            t = 0.5 * ((r < 1 ? 1 : r) - 1);
        }
        *tau = t;
    } else {
        *tau = 0;
    }
    double denom = (double)N - 1.0;
    double vb = m2b / denom;
    double v = m2 / denom;
    *mean = mu;
    *var = v < 0 ? 0 : v;
    *var_binned = vb < 0 ? 0 : vb;
    *stddev = binning ? sqrt(*var_binned / n_bins) : sqrt(*var / N);
}

/* ---------------------------------------------------------------- SR --- */
void orc_sr_moments(const double complex* O, const double complex* E, int N,
                    int P, double complex* d, double complex* F, double* diag) {
    double complex em = 0;
    for (int i = 0; i < N; i++) em += E[i];
    em /= N;
    for (int k = 0; k < P; k++) {
        double complex s = 0, sh = 0;
        for (int i = 0; i < N; i++) {
            s += O[(size_t)i * P + k];
            sh += E[i] * conj(O[(size_t)i * P + k]);
        }
        d[k] = s / N;
        /* F = <E O*> - <E> conj(<O>), stochastic_reconfiguration.cpp:102 */
        F[k] = sh / N - em * conj(d[k]);
        double v = 0;
        for (int i = 0; i < N; i++) {
            double complex q = O[(size_t)i * P + k] - d[k];
            v += creal(q) * creal(q) + cimag(q) * cimag(q);
        }
        diag[k] = v / (N - 1.0);
    }
}

/* S_kl = (1/N) sum_n conj(O_nk) O_nl - conj(d_k) d_l (cg_solver.cpp:274-299) */
void orc_sr_matrix(const double complex* O, const double complex* d, int N,
                   int P, double complex* S) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < P; k++)
        for (int l = 0; l < P; l++) {
            double complex acc = 0;
            for (int i = 0; i < N; i++) acc += conj(O[(size_t)i * P + k]) * O[(size_t)i * P + l];
            S[(size_t)k * P + l] = acc / N - conj(d[k]) * d[l];
        }
}

/* Aprod of cg_solver::solve (non CG_SINGLE branch), cg_solver.cpp:301-318 */
static void aprod(const double complex* O, const double complex* d, double norm,
                  int N, int P, int n_neural, double r1, double r2, double rd,
                  const double* diag, double max_diag, const double complex* b,
                  double complex* x, double complex* tmpN) {
    for (int k = 0; k < P; k++) {
        double f = diag[k] * (k < n_neural ? r1 : r1 + rd) + max_diag * r2;
        x[k] = f * b[k];
    }
    for (int i = 0; i < N; i++) {
        double complex acc = 0;
        for (int k = 0; k < P; k++) acc += O[(size_t)i * P + k] * b[k];
        tmpN[i] = acc;
    }
    double complex db = 0;
    for (int k = 0; k < P; k++) db += d[k] * b[k];
    for (int k = 0; k < P; k++) {
        double complex acc = 0;
        for (int i = 0; i < N; i++) acc += conj(O[(size_t)i * P + k]) * tmpN[i];
        x[k] += acc / norm - conj(d[k]) * db;
    }
}

/* cg_solver::cg1, cg_solver.cpp:119-193 (single process).  Returns the
 * iteration count (the reference's itn_). */
int orc_cg_solve(const double complex* O, const double complex* d, double norm,
                 int N, int P, int n_neural, const double complex* F,
                 double complex* x, double r1, double r2, double rd,
                 const double* diag, int max_iterations, double rtol,
                 double* rs_out) {
    int max_it = max_iterations < 2 * P ? max_iterations : 2 * P;
    if (max_it == 0) max_it = 2 * P;
    if (rtol == 0) rtol = 1e-16;
    double max_diag = diag[0];
    for (int k = 1; k < P; k++)
        if (diag[k] > max_diag) max_diag = diag[k];
    double complex* r = (double complex*)malloc(sizeof(double complex) * P);
    double complex* p = (double complex*)malloc(sizeof(double complex) * P);
    double complex* Ap = (double complex*)malloc(sizeof(double complex) * P);
    double complex* tmp = (double complex*)malloc(sizeof(double complex) * N);
    memcpy(r, F, sizeof(double complex) * P);
    aprod(O, d, norm, N, P, n_neural, r1, r2, rd, diag, max_diag, x, Ap, tmp);
    for (int k = 0; k < P; k++) r[k] -= Ap[k];
    memcpy(p, r, sizeof(double complex) * P);
    double rsold = 0, rs = 0;
    for (int k = 0; k < P; k++) rsold += creal(r[k]) * creal(r[k]) + cimag(r[k]) * cimag(r[k]);
    int itn;
    for (itn = 0; itn < max_it; itn++) {
        aprod(O, d, norm, N, P, n_neural, r1, r2, rd, diag, max_diag, p, Ap, tmp);
        double complex alpha = 0;
        for (int k = 0; k < P; k++) alpha += conj(p[k]) * Ap[k];
        alpha = rsold / alpha;
        rs = 0;
        for (int k = 0; k < P; k++) {
            x[k] += alpha * p[k];
            r[k] -= alpha * Ap[k];
            rs += creal(r[k]) * creal(r[k]) + cimag(r[k]) * cimag(r[k]);
        }
        if (rs < rtol) break;
        for (int k = 0; k < P; k++) p[k] = r[k] + (rs / rsold) * p[k];
        rsold = rs;
    }
    if (rs_out) *rs_out = rs;
    free(r);
    free(p);
    free(Ap);
    free(tmp);
    return itn;
}

/* MINRES-QLP (Choi, Paige & Saunders, SIAM J. Sci. Comput. 33, 2011;
 * ACM TOMS 40, Algorithm 937, 2014), the solver behind optimizer.sr.method =
 * minresqlp: deps/minresqlp/Src/zminresqlpModule.f90:42-1288 driven by
 * minresqlp_adapter.cpp:40-110 (x0 = 0, no preconditioner, the operator
 * with its shift folded in as aprod applies it).  For Hermitian operators
 * the Lanczos coefficients alpha, beta and therefore every rotation and
 * recurrence scalar are real; the vectors are complex.  The iteration runs
 * MINRES updates while the condition estimate Acond stays below trancond
 * and switches to the QLP updates after (minimum-length solutions of
 * near-singular systems).  Stopping rules and their order follow the
 * published routine (istop codes 1-14); maxxnorm, trancond and Acondlim
 * are the adapter's 1e7, 1e7 and 1e15, itnlim 4 P unless given, rtol 1e-16
 * unless given.  Returns the iteration count; rnorm, istop, Acond and the
 * number of QLP iterations through the optional pointers. */
static void symortho_r(double a, double b, double* c, double* s, double* r) {
    const double aa = fabs(a), ab = fabs(b), rmin = 2.2250738585072014e-308;
    if (ab <= rmin) {
        *c = 1, *s = 0, *r = a;
    } else if (aa <= rmin) {
        *c = 0, *s = 1, *r = b;
    } else if (ab > aa) {
        const double t = aa / ab;
        double cc = 1.0 / sqrt(1.0 + t * t);
        *s = cc * ((b > 0) == (a > 0) ? 1.0 : -1.0);
        *c = cc * t;
        *r = b / *s;
    } else {
        const double t = ab / aa;
        const double cc = 1.0 / sqrt(1.0 + t * t);
        *c = cc;
        *s = cc * t * ((b > 0) == (a > 0) ? 1.0 : -1.0);
        *r = a / cc;
    }
}

static double nrm(int n, const double* v) {
    double s = 0;
    for (int i = 0; i < n; i++) s += v[i] * v[i];
    return sqrt(s);
}

int orc_minresqlp_solve(const double complex* O, const double complex* d, double norm,
                        int N, int P, int n_neural, const double complex* F,
                        double complex* x, double r1, double r2, double rd,
                        const double* diag, int max_iterations, double rtol,
                        double* rnorm_out, int* istop_out, double* acond_out, int* qlp_out) {
    const double eps = 2.220446049250313e-16, maxxnorm = 1e7, trancond = 1e7, Acondlim = 1e15;
    const int itnlim = max_iterations > 0 ? max_iterations : 4 * P;
    if (rtol <= 0) rtol = 1e-16;
    double max_diag = diag[0];
    for (int k = 1; k < P; k++)
        if (diag[k] > max_diag) max_diag = diag[k];
    size_t sz = sizeof(double complex) * P;
    double complex *v = malloc(sz), *y = malloc(sz), *R1 = malloc(sz), *R2 = malloc(sz);
    double complex *w = calloc(P, sizeof(double complex)), *wl = calloc(P, sizeof(double complex));
    double complex *wl2 = calloc(P, sizeof(double complex)), *xl2 = calloc(P, sizeof(double complex));
    double complex* tmp = malloc(sizeof(double complex) * N);
    for (int k = 0; k < P; k++) x[k] = 0;
    memcpy(y, F, sz);
    memcpy(R1, F, sz);
    memcpy(R2, F, sz);
    double beta1 = 0;
    for (int k = 0; k < P; k++) beta1 += creal(F[k]) * creal(F[k]) + cimag(F[k]) * cimag(F[k]);
    int istop = beta1 == 0 ? 3 : 0;
    beta1 = sqrt(beta1);
    const double ieps = 0.1 / eps;
    int itn = 0, qlp = 0, lastiter = 0;
    double beta = 0, betal, betan = beta1, alfa, pnorm = 0;
    double dbar, dlta = 0, epln, eplnn = 0, dltan = 0, gbar = 0, dlta_qlp;
    double gama = 0, gamal = 0, gamal2 = 0, gamal3, gama_tmp;
    double tau = 0, taul = 0, taul2, phi = beta1, cs = -1, sn = 0, cr1 = -1, sr1 = 0, cr2 = -1, sr2 = 0;
    double vepln = 0, veplnl = 0, veplnl2 = 0, eta = 0, etal = 0, etal2 = 0;
    double u = 0, ul = 0, ul2 = 0, ul3 = 0, ul4;
    double xnorm = 0, xl2norm = 0, Axnorm = 0, Anorm = 0, Acond = 1, Acondl = 1, gmin = 0, gminl = 0, gminl2;
    double rnorm = beta1, rnorml = beta1, relres = 1, relresl = 0, relAresl = 0, t1 = 2, t2 = 2;
    double gamal_qlp = 0, vepln_qlp = 0, gama_qlp = 0, ul_qlp = 0, u_qlp = 0;
    while (istop <= 0) {
        itn++;
        // Lanczos: v = y / beta, y = A v - (beta / betal) r1 - (alfa / beta) r2
        betal = beta;
        beta = betan;
        for (int k = 0; k < P; k++) v[k] = y[k] / beta;
        aprod(O, d, norm, N, P, n_neural, r1, r2, rd, diag, max_diag, v, y, tmp);
        if (itn >= 2)
            for (int k = 0; k < P; k++) y[k] -= (beta / betal) * R1[k];
        alfa = 0;
        for (int k = 0; k < P; k++) alfa += creal(conj(v[k]) * y[k]);
        for (int k = 0; k < P; k++) y[k] -= (alfa / beta) * R2[k];
        memcpy(R1, R2, sz);
        memcpy(R2, y, sz);
        betan = 0;
        for (int k = 0; k < P; k++) betan += creal(y[k]) * creal(y[k]) + cimag(y[k]) * cimag(y[k]);
        betan = sqrt(betan);
        {
            const double q2[2] = {alfa, betan}, q3[3] = {beta, alfa, betan};
            pnorm = itn == 1 ? nrm(2, q2) : nrm(3, q3);
        }
        // previous left reflection
        dbar = dltan;
        dlta = cs * dbar + sn * alfa;
        epln = eplnn;
        gbar = sn * dbar - cs * alfa;
        eplnn = sn * betan;
        dltan = -cs * betan;
        dlta_qlp = dlta;
        // current left reflection
        gamal3 = gamal2;
        gamal2 = gamal;
        gamal = gama;
        symortho_r(gbar, betan, &cs, &sn, &gama);
        gama_tmp = gama;
        taul2 = taul;
        taul = tau;
        tau = cs * phi;
        phi = sn * phi;
        Axnorm = sqrt(Axnorm * Axnorm + tau * tau);
        // previous right reflection P_{k-2,k}
        if (itn > 2) {
            veplnl2 = veplnl;
            etal2 = etal;
            etal = eta;
            const double dt = sr2 * vepln - cr2 * dlta;
            veplnl = cr2 * vepln + sr2 * dlta;
            dlta = dt;
            eta = sr2 * gama;
            gama = -cr2 * gama;
        }
        // current right reflection P_{k-1,k}
        if (itn > 1) {
            double g;
            symortho_r(gamal, dlta, &cr1, &sr1, &g);
            gamal = g;
            vepln = sr1 * gama;
            gama = -cr1 * gama;
        }
        // xnorm
        ul4 = ul3;
        ul3 = ul2;
        if (itn > 2) ul2 = (taul2 - etal2 * ul4 - veplnl2 * ul3) / gamal2;
        if (itn > 1) ul = (taul - etal * ul3 - veplnl * ul2) / gamal;
        {
            const double q3[3] = {xl2norm, ul2, ul};
            const double xt = nrm(3, q3);
            if (fabs(gama) > 0 && xt < maxxnorm) {
                u = (tau - eta * ul2 - vepln * ul) / gama;
                const double q2[2] = {xt, u};
                if (relAresl < relresl && nrm(2, q2) > maxxnorm) {
                    u = 0;
                    istop = 12;
                }
            } else {
                u = 0;
                istop = 14;
            }
        }
        {
            const double q2[2] = {xl2norm, ul2};
            xl2norm = nrm(2, q2);
            const double q3[3] = {xl2norm, ul, u};
            xnorm = nrm(3, q3);
        }
        if (Acond < trancond && istop == 0 && qlp == 0) {
            // MINRES updates
            for (int k = 0; k < P; k++) {
                const double complex a = wl[k];
                wl2[k] = a;
                wl[k] = w[k];
                if (fabs(gama_tmp) > 0) w[k] = (v[k] - epln * wl2[k] - dlta_qlp * wl[k]) / gama_tmp;
            }
            if (xnorm < maxxnorm) {
                for (int k = 0; k < P; k++) x[k] += tau * w[k];
            } else {
                istop = 12;
                lastiter = 1;
            }
        } else {
            // MINRES-QLP updates
            qlp++;
            if (qlp == 1) {
                for (int k = 0; k < P; k++) xl2[k] = 0;
                if (itn > 1) {
                    for (int k = 0; k < P; k++) {
                        if (itn > 3) wl2[k] = gamal3 * wl2[k] + veplnl2 * wl[k] + etal * w[k];
                        if (itn > 2) wl[k] = gamal_qlp * wl[k] + vepln_qlp * w[k];
                        w[k] = gama_qlp * w[k];
                        xl2[k] = x[k] - ul_qlp * wl[k] - u_qlp * w[k];
                    }
                }
            }
            for (int k = 0; k < P; k++) {
                if (itn == 1) {
                    wl2[k] = wl[k];
                    wl[k] = sr1 * v[k];
                    w[k] = -cr1 * v[k];
                } else if (itn == 2) {
                    wl2[k] = wl[k];
                    wl[k] = cr1 * w[k] + sr1 * v[k];
                    w[k] = sr1 * w[k] - cr1 * v[k];
                } else {
                    wl2[k] = wl[k];
                    wl[k] = w[k];
                    w[k] = sr2 * wl2[k] - cr2 * v[k];
                    wl2[k] = cr2 * wl2[k] + sr2 * v[k];
                    v[k] = cr1 * wl[k] + sr1 * w[k];
                    w[k] = sr1 * wl[k] - cr1 * w[k];
                    wl[k] = v[k];
                }
                xl2[k] += ul2 * wl2[k];
                x[k] = xl2[k] + ul * wl[k] + u * w[k];
            }
        }
        // next right reflection P_{k-1,k+1}
        {
            const double gt = gamal;
            symortho_r(gt, eplnn, &cr2, &sr2, &gamal);
            gamal_qlp = gt;
        }
        vepln_qlp = vepln;
        gama_qlp = gama;
        ul_qlp = ul;
        u_qlp = u;
        // norm and condition estimates
        const double ag = fabs(gama);
        Anorm = fmax(fmax(Anorm, pnorm), fmax(fabs(gamal), ag));
        if (itn == 1) {
            gmin = ag;
            gminl = gmin;
        } else {
            gminl2 = gminl;
            gminl = gmin;
            gmin = fmin(gminl2, fmin(fabs(gamal), ag));
        }
        Acondl = Acond;
        Acond = Anorm / gmin;
        rnorml = rnorm;
        relresl = relres;
        if (istop != 14) rnorm = fabs(phi);
        relres = rnorm / (Anorm * xnorm + beta1);
        {
            const double q2[2] = {gbar, dltan};
            const double rootl = nrm(2, q2);
            relAresl = rootl / Anorm;
        }
        // stopping rules, in the published order
        const double epsx = Anorm * xnorm * eps;
        if (istop == 0 || istop == 14) {
            t1 = 1 + relres;
            t2 = 1 + relAresl;
        }
        if (t1 <= 1) istop = 5;
        else if (t2 <= 1) istop = 7;
        else if (relres <= rtol) istop = 4;
        else if (relAresl <= rtol) istop = 6;
        else if (epsx >= beta1) istop = 2;
        else if (xnorm >= maxxnorm) istop = 12;
        else if (Acond >= Acondlim || Acond >= ieps) istop = 13;
        else if (itn >= itnlim) istop = 8;
        else if (betan < eps) istop = 1;
        if (istop == 6 || istop == 7 || istop == 12 || istop == 13) lastiter = 1;
        if (istop != 0 && lastiter) {
            itn--;
            Acond = Acondl;
            rnorm = rnorml;
            relres = relresl;
        }
    }
    if (rnorm_out) *rnorm_out = rnorm;
    if (istop_out) *istop_out = istop;
    if (acond_out) *acond_out = Acond;
    if (qlp_out) *qlp_out = qlp;
    free(v), free(y), free(R1), free(R2), free(w), free(wl), free(wl2), free(xl2), free(tmp);
    return itn;
}

/* decay_t, abstract_optimizer.cpp:27-54 */
void orc_decay_init(orc_decay* d, double initial, double min, double decay,
                    uint64_t offset) {
    d->initial = initial;
    d->min = min;
    d->decay = decay;
    d->value = pow(decay, (double)offset) * initial;
    d->min_reached = decay == 1.0;
}

double orc_decay_get(orc_decay* d) {
    if (!d->min_reached) {
        d->value *= d->decay;
        if (d->value < d->min) {
            d->min_reached = 1;
            d->value = d->min;
        }
    }
    return d->value;
}
