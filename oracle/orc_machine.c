/*
 * orc_machine.c -- oracle restatement of the reference's wavefunctions:
 * machine/rbm_base.cpp, machine/rbm_symmetry.cpp, machine/pfaffian.cpp,
 * math.cpp, operators/local_op.cpp (TEST INFRASTRUCTURE ONLY; see orc.h).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "orc.h"

static inline int bit(const uint32_t* s, int i) { return (s[i >> 5] >> (i & 31)) & 1; }
static inline double sig(const uint32_t* s, int i) { return bit(s, i) ? -1.0 : 1.0; }

int orc_n_neural(const orc_machine* m) {
    /* rbm_base.cpp:40  n_vb + (alpha + alpha*n) * n_vb  == n_vb + nh + n*nh */
    return m->n_vb + m->nh + m->n * m->nh;
}

int orc_n_params(const orc_machine* m) {
    return orc_n_neural(m) + (m->has_pf ? 4 * m->n_indep : 0);
}

/* theta[k + nh*s] = h_k + sum_i sigma_i W[P_s(i), k]
 * (rbm_base.cpp:161-172, rbm_symmetry.cpp:48-61) */
void orc_theta(const orc_machine* m, const uint32_t* spins, double complex* th) {
    int n = m->n, nh = m->nh;
    for (int s = 0; s < m->S; s++)
        for (int k = 0; k < nh; k++) {
            double complex acc = m->h[k];
            for (int i = 0; i < n; i++) {
                int p = m->perm ? m->perm[s * n + i] : i;
                acc += sig(spins, i) * m->W[p + n * k];
            }
            th[k + nh * s] = acc;
        }
}

/* Numerically safe sum of ln cosh, math.cpp:37-56 */
double complex orc_lncosh_sum(const double complex* x, int len) {
    double gre = 0, gim = 0;
    for (int i = 0; i < len; i++) {
        double a = creal(x[i]);
        double reabs = fabs(a);
        double lre = reabs - M_LN2;
        reabs = exp(-2.0 * reabs);
        lre += log1p(reabs);
        double si = sin(cimag(x[i]));
        double co = cos(cimag(x[i]));
        si *= copysign((1.0 - reabs) / (1.0 + reabs), a);
        lre += 0.5 * log(si * si + co * co);
        gre += lre;
        gim += atan2(si, co);
    }
    return gre + I * gim;
}

static double complex bias_part(const orc_machine* m, const uint32_t* spins) {
    double complex acc = 0;
    if (!m->symmetric) {
        /* rbm_base.cpp:294-296 */
        for (int i = 0; i < m->n_vb; i++) acc += m->v[i] * sig(spins, i);
    } else {
        /* rbm_symmetry.cpp:138-147 */
        for (int i = 0; i < m->n_vb; i++)
            for (int s = 0; s < m->S; s++)
                acc += m->v[i] * sig(spins, m->perm[s * m->n + m->basis[i]]);
    }
    return acc;
}

/* ------------------------------------------------------------ Pfaffian -- */
/* pfaffian.cpp:31-85: independent-parameter index matrix (row-major here,
 * bs[i*n + j] == Eigen bs_(i, j)).  Returns n_indep = max entry. */
int orc_pfaffian_bs(int n, int S, const int* perm, int n_basis,
                    const int* basis, int* bs) {
    memset(bs, 0, sizeof(int) * n * n);
    int offset = 0;
    for (int bi = 0; bi < n_basis; bi++) {
        for (int s = 0; s < S; s++) {
            const int* idcs = perm + s * n;
            int f = idcs[0] > idcs[1] ? -1 : 1;
            for (int j = 0; j < n; j++) {
                int a = idcs[basis[bi]];
                int b = idcs[j];
                if (b == a)
                    bs[b * n + a] = 0;
                else
                    bs[b * n + a] = f * (j + offset);
            }
        }
        offset += n;
    }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < i; j++) {
            if (abs(bs[i * n + j]) <= abs(bs[j * n + i]))
                bs[j * n + i] = -bs[i * n + j];
            else
                bs[i * n + j] = -bs[j * n + i];
        }
    int mx = 0;
    for (int i = 0; i < n * n; i++)
        if (bs[i] > mx) mx = bs[i];
    /* condense indices (pfaffian.cpp:67-73); the loop bound is re-read each
     * iteration, exactly as Eigen's maxCoeff() in the loop condition */
    for (int i = 1;; i++) {
        mx = 0;
        for (int q = 0; q < n * n; q++)
            if (bs[q] > mx) mx = bs[q];
        if (!(i < mx)) break;
        for (;;) {
            int cnt = 0;
            for (int q = 0; q < n * n; q++) cnt += bs[q] == i;
            if (cnt != 0) break;
            for (int q = 0; q < n * n; q++) {
                if (bs[q] > i)
                    bs[q] -= 1;
                else if (bs[q] < -i)
                    bs[q] += 1;
            }
        }
    }
    mx = 0;
    for (int q = 0; q < n * n; q++)
        if (bs[q] > mx) mx = bs[q];
    return mx;
}

/* pfaffian::a, pfaffian.cpp:127-137 */
static double complex pf_a(const orc_machine* m, const uint32_t* st, int i, int j,
                           int fi, int fj) {
    if (i == j) return 0;
    int n = m->n;
    int b = m->bs[i * n + j];
    double sgn = b < 0 ? -1.0 : 1.0;
    int sp = (j < i) ? (((bit(st, i) ^ fi) << 1) + (bit(st, j) ^ fj))
                     : (((bit(st, j) ^ fj) << 1) + (bit(st, i) ^ fi));
    return sgn * m->fs[(abs(b) - 1) + m->n_indep * sp];
}

/* pfaffian::get_mat, pfaffian.cpp:270-282 (column-major X[i + n*j]) */
void orc_pf_matrix(const orc_machine* m, const uint32_t* spins, double complex* X) {
    int n = m->n;
    for (int i = 0; i < n; i++) {
        X[i + n * i] = 0;
        for (int j = 0; j < i; j++) {
            double complex v = pf_a(m, spins, i, j, 0, 0);
            X[i + n * j] = v;
            X[j + n * i] = -v;
        }
    }
}

/* Pfaffian of an antisymmetric matrix by Parlett-Reid tridiagonalisation
 * with partial pivoting (Wimmer, ACM TOMS 38 (2012) Algorithm 923; the
 * reference calls PFAPACK skpf10_z(..., "L", "P"), math.hpp:109-114).
 * A is column-major and overwritten; result = mantissa * 10^exp10. */
double complex orc_pfaffian10(int n, double complex* A, int* exp10) {
    double complex mant = 1;
    int e10 = 0;
    if (n % 2) {
        *exp10 = 0;
        return 0;
    }
#define A_(r, c) A[(r) + (size_t)n * (c)]
    for (int k = 0; k < n - 1; k += 2) {
        int kp = k + 1;
        double best = cabs(A_(k + 1, k));
        for (int i = k + 2; i < n; i++)
            if (cabs(A_(i, k)) > best) {
                best = cabs(A_(i, k));
                kp = i;
            }
        if (kp != k + 1) {
            for (int c = 0; c < n; c++) {
                double complex t = A_(k + 1, c);
                A_(k + 1, c) = A_(kp, c);
                A_(kp, c) = t;
            }
            for (int r = 0; r < n; r++) {
                double complex t = A_(r, k + 1);
                A_(r, k + 1) = A_(r, kp);
                A_(r, kp) = t;
            }
            mant = -mant;
        }
        if (A_(k + 1, k) == 0) {
            *exp10 = 0;
            return 0;
        }
        mant *= A_(k, k + 1);
        if (mant != 0) {
            int s = (int)floor(log10(cabs(mant)));
            mant *= pow(10.0, -s);
            e10 += s;
        }
        if (k + 2 < n) {
            /* tau_i = A(k, i) / A(k, k+1), i >= k+2; rank-2 update of the
             * trailing block keeping it antisymmetric */
            double complex piv = A_(k, k + 1);
            for (int i = k + 2; i < n; i++) {
                double complex ti = A_(k, i) / piv;
                for (int j = k + 2; j < n; j++) {
                    double complex tj = A_(k, j) / piv;
                    A_(i, j) += ti * A_(j, k + 1) - A_(i, k + 1) * tj;
                }
            }
        }
    }
#undef A_
    *exp10 = e10;
    return mant;
}

/* Dense complex inverse by Gauss-Jordan with partial pivoting (column-major).
 * Stands in for Eigen's complete-orthogonal-decomposition pseudo-inverse
 * (pfaffian.cpp:289) on the non-singular X the tests use. */
static int cinv(int n, const double complex* A, double complex* Ainv) {
    double complex* M = (double complex*)malloc(sizeof(double complex) * n * 2 * n);
#define M_(r, c) M[(r) + (size_t)n * (c)]
    for (int r = 0; r < n; r++)
        for (int c = 0; c < n; c++) {
            M_(r, c) = A[r + n * c];
            M_(r, c + n) = r == c ? 1 : 0;
        }
    for (int c = 0; c < n; c++) {
        int p = c;
        for (int r = c + 1; r < n; r++)
            if (cabs(M_(r, c)) > cabs(M_(p, c))) p = r;
        if (M_(p, c) == 0) {
            free(M);
            return -1;
        }
        if (p != c)
            for (int q = 0; q < 2 * n; q++) {
                double complex t = M_(c, q);
                M_(c, q) = M_(p, q);
                M_(p, q) = t;
            }
        double complex iv = 1.0 / M_(c, c);
        for (int q = 0; q < 2 * n; q++) M_(c, q) *= iv;
        for (int r = 0; r < n; r++)
            if (r != c && M_(r, c) != 0) {
                double complex f = M_(r, c);
                for (int q = 0; q < 2 * n; q++) M_(r, q) -= f * M_(c, q);
            }
    }
    for (int r = 0; r < n; r++)
        for (int c = 0; c < n; c++) Ainv[r + n * c] = M_(r, c + n);
#undef M_
    free(M);
    return 0;
}

/* pfaffian::get_context, pfaffian.cpp:284-297 */
void orc_pf_context(const orc_machine* m, const uint32_t* spins, orc_pfctx* c) {
    int n = m->n;
    double complex* X = (double complex*)malloc(sizeof(double complex) * n * n);
    orc_pf_matrix(m, spins, X);
    cinv(n, X, c->inv);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < i; j++) {
            double complex a = 0.5 * (c->inv[i + n * j] - c->inv[j + n * i]);
            c->inv[i + n * j] = a;
            c->inv[j + n * i] = -a;
        }
    for (int i = 0; i < n; i++) c->inv[i + n * i] = 0;
    c->pf_mant = orc_pfaffian10(n, X, &c->pf_exp10);
    c->update_factor = 1;
    free(X);
}

/* pfaffian::update_context (updating branch), pfaffian.cpp:314-397 */
void orc_pf_update(const orc_machine* m, const uint32_t* st, const int* flips,
                   int mm, orc_pfctx* c) {
    if (mm == 0) return;
    int n = m->n, m2 = 2 * mm;
    double sign = ((mm * (mm + 1) / 2) % 2 == 0) ? 1.0 : -1.0;
    double complex* B = (double complex*)calloc((size_t)n * m2, sizeof(double complex));
    double complex* Ci = (double complex*)calloc((size_t)m2 * m2, sizeof(double complex));
    double complex* IB = (double complex*)calloc((size_t)n * m2, sizeof(double complex));
    char* fl = (char*)calloc(n, 1);
    for (int q = 0; q < mm; q++) fl[flips[q]] = 1;
#define B_(r, c) B[(r) + (size_t)n * (c)]
#define C_(r, c) Ci[(r) + (size_t)m2 * (c)]
    for (int q = 0; q < mm; q++) C_(mm + q, q) = 1;
    for (int k = 0; k < mm; k++) {
        B_(flips[k], mm + k) = 1;
        for (int i = 0; i < n; i++)
            if (flips[k] != i)
                B_(i, k) = pf_a(m, st, i, flips[k], fl[i], 1) - pf_a(m, st, i, flips[k], 0, 0);
        for (int l = 0; l < k; l++)
            C_(k, l) = -pf_a(m, st, flips[k], flips[l], 1, 1) + pf_a(m, st, flips[k], flips[l], 0, 0);
    }
    for (int r = 0; r < m2; r++)
        for (int q = r + 1; q < m2; q++) C_(r, q) = -C_(q, r);
    /* invB = inv * B */
    for (int r = 0; r < n; r++)
        for (int q = 0; q < m2; q++) {
            double complex acc = 0;
            for (int t = 0; t < n; t++) acc += c->inv[r + n * t] * B_(t, q);
            IB[r + (size_t)n * q] = acc;
        }
    /* tmp = 0.5 * B^T invB;  Cinv += tmp - tmp^T */
    double complex* tmp = (double complex*)calloc((size_t)m2 * m2, sizeof(double complex));
    for (int r = 0; r < m2; r++)
        for (int q = 0; q < m2; q++) {
            double complex acc = 0;
            for (int t = 0; t < n; t++) acc += B_(t, r) * IB[t + (size_t)n * q];
            tmp[r + m2 * q] = 0.5 * acc;
        }
    for (int r = 0; r < m2; r++)
        for (int q = 0; q < m2; q++) C_(r, q) += tmp[r + m2 * q] - tmp[q + m2 * r];
    /* C = 0.5 Cinv^{-1}; C -= C^T */
    double complex* Cm = (double complex*)calloc((size_t)m2 * m2, sizeof(double complex));
    cinv(m2, Ci, Cm);
    double complex* Ca = (double complex*)calloc((size_t)m2 * m2, sizeof(double complex));
    for (int r = 0; r < m2; r++)
        for (int q = 0; q < m2; q++) Ca[r + m2 * q] = 0.5 * Cm[r + m2 * q] - 0.5 * Cm[q + m2 * r];
    /* inv += 0.5 (invB C invB^T) - (.)^T */
    double complex* T1 = (double complex*)calloc((size_t)n * m2, sizeof(double complex));
    for (int r = 0; r < n; r++)
        for (int q = 0; q < m2; q++) {
            double complex acc = 0;
            for (int t = 0; t < m2; t++) acc += IB[r + (size_t)n * t] * Ca[t + m2 * q];
            T1[r + (size_t)n * q] = acc;
        }
    double complex* T2 = (double complex*)calloc((size_t)n * n, sizeof(double complex));
    for (int r = 0; r < n; r++)
        for (int q = 0; q < n; q++) {
            double complex acc = 0;
            for (int t = 0; t < m2; t++) acc += T1[r + (size_t)n * t] * IB[q + (size_t)n * t];
            T2[r + (size_t)n * q] = 0.5 * acc;
        }
    for (int r = 0; r < n; r++)
        for (int q = 0; q < n; q++) c->inv[r + n * q] += T2[r + n * q] - T2[q + n * r];
    int e;
    double complex c2 = orc_pfaffian10(m2, Ci, &e) * sign;
    c->pf_mant *= c2;
    c->pf_exp10 += e;
    c->update_factor = c2 * pow(10.0, e);
    int s = (int)log10(cabs(c->pf_mant));
    if (abs(s) > 1) {
        c->pf_mant *= pow(10.0, -s);
        c->pf_exp10 += s;
    }
#undef B_
#undef C_
    free(B);
    free(Ci);
    free(IB);
    free(fl);
    free(tmp);
    free(Cm);
    free(Ca);
    free(T1);
    free(T2);
}

/* --------------------------------------------------------------- psi --- */
static double complex log_pf(const orc_machine* m, const uint32_t* spins) {
    int n = m->n;
    double complex* X = (double complex*)malloc(sizeof(double complex) * n * n);
    orc_pf_matrix(m, spins, X);
    int e;
    double complex p = orc_pfaffian10(n, X, &e);
    free(X);
    return clog(p) + e * M_LN10;
}

/* log psi = bias + sum lncosh(theta) (+ log Pf), rbm_base.cpp:294-304 and
 * pfaffian.hpp:73-75 */
double complex orc_log_psi(const orc_machine* m, const uint32_t* spins) {
    int T = m->nh * m->S;
    double complex* th = (double complex*)malloc(sizeof(double complex) * T);
    orc_theta(m, spins, th);
    double complex r = bias_part(m, spins) + orc_lncosh_sum(th, T);
    free(th);
    if (m->has_pf) r += log_pf(m, spins);
    return r;
}

/* log_psi_over_psi + log_psi_over_psi_bias, rbm_base.cpp:306-344, with
 * theta' = theta - 2 sigma_f W[P_s(f)] (rbm_base.cpp:174-192,
 * rbm_symmetry.cpp:63-95); the Pfaffian factor is Pf(X')/Pf(X). */
double complex orc_log_psi_over_psi(const orc_machine* m, const uint32_t* spins,
                                    const int* flips, int nf) {
    if (nf == 0) return 0;
    int n = m->n, nh = m->nh, T = nh * m->S;
    double complex r = 0;
    for (int q = 0; q < nf; q++) r -= 2.0 * sig(spins, flips[q]) * m->v[flips[q] % m->n_vb];
    double complex* th = (double complex*)malloc(sizeof(double complex) * T);
    double complex* th2 = (double complex*)malloc(sizeof(double complex) * T);
    orc_theta(m, spins, th);
    memcpy(th2, th, sizeof(double complex) * T);
    for (int s = 0; s < m->S; s++)
        for (int q = 0; q < nf; q++) {
            int f = flips[q];
            int p = m->perm ? m->perm[s * n + f] : f;
            double sf = sig(spins, f);
            for (int k = 0; k < nh; k++) th2[k + nh * s] -= 2.0 * sf * m->W[p + n * k];
        }
    r += orc_lncosh_sum(th2, T) - orc_lncosh_sum(th, T);
    free(th);
    free(th2);
    if (m->has_pf) {
        uint32_t s2[4] = {spins[0], spins[1], spins[2], spins[3]};
        for (int q = 0; q < nf; q++) s2[flips[q] >> 5] ^= 1u << (flips[q] & 31);
        r += log_pf(m, s2) - log_pf(m, spins);
    }
    return r;
}

/* derivative: rbm_base.cpp:194-217, rbm_symmetry.cpp:97-130,
 * pfaffian.cpp:399-415 */
void orc_derivative(const orc_machine* m, const uint32_t* spins, double complex* O) {
    int n = m->n, nh = m->nh, S = m->S, T = nh * S;
    int P = orc_n_params(m);
    memset(O, 0, sizeof(double complex) * P);
    double complex* th = (double complex*)malloc(sizeof(double complex) * T);
    orc_theta(m, spins, th);
    for (int t = 0; t < T; t++) th[t] = ctanh(th[t]);
    if (!m->symmetric) {
        for (int i = 0; i < m->n_vb; i++) O[i] = sig(spins, i);
        for (int k = 0; k < nh; k++) O[m->n_vb + k] = th[k];
        for (int k = 0; k < nh; k++)
            for (int j = 0; j < n; j++) O[m->n_vb + nh + j + n * k] = sig(spins, j) * th[k];
    } else {
        int* inv = (int*)malloc(sizeof(int) * S * n);
        for (int s = 0; s < S; s++)
            for (int i = 0; i < n; i++) inv[s * n + m->perm[s * n + i]] = i;
        for (int i = 0; i < m->n_vb; i++)
            for (int s = 0; s < S; s++) O[i] += sig(spins, m->perm[s * n + m->basis[i]]);
        for (int k = 0; k < nh; k++)
            for (int s = 0; s < S; s++) O[m->n_vb + k] += th[k + nh * s];
        for (int s = 0; s < S; s++)
            for (int k = 0; k < nh; k++)
                for (int j = 0; j < n; j++)
                    O[m->n_vb + nh + j + n * k] += sig(spins, inv[s * n + j]) * th[k + nh * s];
        free(inv);
    }
    free(th);
    if (m->has_pf) {
        orc_pfctx c;
        c.inv = (double complex*)malloc(sizeof(double complex) * n * n);
        orc_pf_context(m, spins, &c);
        double complex* d = O + orc_n_neural(m);
        for (int i = 0; i < n; i++)
            for (int j = 0; j < i; j++) {
                double complex x = c.inv[i + n * j];
                int b = m->bs[i * n + j];
                int sp = (bit(spins, i) << 1) + bit(spins, j);
                d[(abs(b) - 1) + m->n_indep * sp] += b > 0 ? -x : x;
            }
        free(c.inv);
    }
}

/* local_op::evaluate summed over the Hamiltonian chain,
 * operators/local_op.cpp:31-60, local_op_chain.cpp:54-60 */
double complex orc_eloc(const orc_machine* m, const orc_ops* ops, const uint32_t* spins) {
    double complex E = 0;
    for (int o = 0; o < ops->n_ops; o++) {
        int k = ops->k[o];
        const int* as = ops->sites + 6 * o;
        int d = 1 << k;
        int loc = 0;
        for (int i = 0; i < k; i++)
            if (bit(spins, as[i])) loc |= 1 << i;
        const double* row = ops->mats + 2 * ((size_t)ops->mat_off[o] + (size_t)loc * d);
        double complex res = 0;
        for (int c = 0; c < d; c++) {
            double complex val = row[2 * c] + I * row[2 * c + 1];
            if (val == 0) continue;
            if (c == loc) {
                res += val;
            } else {
                int fl[6], nf = 0;
                int x = c ^ loc;
                for (int i = 0; i < k; i++)
                    if ((x >> i) & 1) fl[nf++] = as[i];
                res += val * cexp(orc_log_psi_over_psi(m, spins, fl, nf));
            }
        }
        E += res;
    }
    return E;
}

void orc_eval_batch(const orc_machine* m, const orc_ops* ops, const uint32_t* spins,
                    int B, double complex* logpsi, double complex* eloc,
                    double complex* O) {
    int P = orc_n_params(m);
#pragma omp parallel for schedule(dynamic, 4)
    for (int b = 0; b < B; b++) {
        const uint32_t* s = spins + 4 * b;
        if (logpsi) logpsi[b] = orc_log_psi(m, s);
        if (eloc) eloc[b] = orc_eloc(m, ops, s);
        if (O) orc_derivative(m, s, O + (size_t)b * P);
    }
}
