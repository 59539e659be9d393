// ed.cu -- exact diagonalisation of a model's Hamiltonian on the GPU: the
// lowest eigenvalue (and optionally its eigenvector) by the Lanczos method
// on the full 2^n basis.  It cross-checks the variational energies on
// systems the CPU cannot diagonalise (up to 28 sites; the reference only
// diagonalises small systems in Python with scipy, python_adapter/rbm/
// __init__.py:16-41, whose basis convention is used: site i <-> bit i of
// the basis index, <x|H|y> = op[loc(x)][loc(y)]).
//
// H v is applied in gather form from the same operator tables the E_loc
// kernels use: (H v)[s] = sum_ops sum_q val_q v[s ^ flip_q(s)], one thread
// per basis state (deterministic, no atomics).  Dot products reduce in a
// fixed order.  Plain Lanczos (no reorthogonalisation): the lowest Ritz
// value converges first and is unaffected by the loss of orthogonality
// that produces spurious copies of converged eigenvalues.  The tridiagonal
// problem is solved on the host by Sturm-sequence bisection; the
// eigenvector, when asked for, by inverse iteration on the tridiagonal
// matrix and a second Lanczos pass that accumulates the basis vectors.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "ed.cuh"

namespace rbmnqs {
namespace {

constexpr int kThreads = 256;
constexpr int kBlocks = 592;

__global__ void ed_apply(HamDev H, int64_t N, const double2* __restrict__ v, double2* __restrict__ w) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < N; s += (int64_t)gridDim.x * blockDim.x) {
        double ax = 0, ay = 0;
        for (int o = 0; o < H.n_ops; o++) {
            const OpDev* op = H.ops + o;
            const int k = op->k;
            int loc = 0;
            for (int i = 0; i < k; i++) loc |= (int)((s >> op->sites[i]) & 1) << i;
            const int q0 = __ldg(H.rowptr + op->rp + loc), q1 = __ldg(H.rowptr + op->rp + loc + 1);
            for (int q = q0; q < q1; q++) {
                const uint32_t mask = __ldg(H.ent_mask + q);
                const double2 val = __ldg(H.ent_val + q);
                int64_t t = s;
                for (int i = 0; i < k; i++)
                    if ((mask >> i) & 1) t ^= int64_t(1) << op->sites[i];
                const double2 x = __ldg(v + t);
                ax += val.x * x.x - val.y * x.y;
                ay += val.x * x.y + val.y * x.x;
            }
        }
        w[s] = make_double2(ax, ay);
    }
}

__device__ __forceinline__ double bsum(double v, double* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double r = red[0];
    for (int i = 1; i < nw; i++) r += red[i];
    __syncthreads();
    return r;
}

// partial sums of conj(a) . b per block
__global__ void ed_dot(const double2* a, const double2* b, int64_t N, double2* part) {
    __shared__ double red[32];
    double sx = 0, sy = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 x = a[i], y = b[i];
        sx += x.x * y.x + x.y * y.y;
        sy += x.x * y.y - x.y * y.x;
    }
    sx = bsum(sx, red);
    sy = bsum(sy, red);
    if (threadIdx.x == 0) part[blockIdx.x] = make_double2(sx, sy);
}

__global__ void ed_sum(const double2* part, int G, double2* out) {
    if (threadIdx.x == 0) {
        double2 s = make_double2(0, 0);
        for (int i = 0; i < G; i++) {
            s.x += part[i].x;
            s.y += part[i].y;
        }
        *out = s;
    }
}

// w = (w - alpha v - beta u) / norm as needed by the three-term recurrence:
// mode 0: w -= alpha v + beta u; mode 1: v_next = w / beta (into u)
__global__ void ed_axpy(double2* w, const double2* v, const double2* u, double alpha, double beta, int64_t N) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        double2 x = w[i];
        const double2 a = v[i];
        x.x -= alpha * a.x;
        x.y -= alpha * a.y;
        if (u) {
            const double2 b = u[i];
            x.x -= beta * b.x;
            x.y -= beta * b.y;
        }
        w[i] = x;
    }
}

__global__ void ed_scale(const double2* w, double f, double2* out, int64_t N) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = make_double2(w[i].x * f, w[i].y * f);
}

__global__ void ed_accumulate(double2* psi, const double2* v, double c, int64_t N) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        psi[i].x += c * v[i].x;
        psi[i].y += c * v[i].y;
    }
}

// deterministic start vector: splitmix64 of (seed, index) -> two uniforms
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}
__global__ void ed_start(double2* v, int64_t N, uint64_t seed) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t a = mix64(seed ^ mix64((uint64_t)i)), b = mix64(a);
        v[i] = make_double2((double)(a >> 11) * 0x1.0p-53 - 0.5, (double)(b >> 11) * 0x1.0p-53 - 0.5);
    }
}

// number of eigenvalues of the symmetric tridiagonal (a, b) below x
int sturm_count(const std::vector<double>& a, const std::vector<double>& b, int m, double x) {
    int c = 0;
    double q = 1.0;
    for (int i = 0; i < m; i++) {
        const double off = i ? b[i - 1] * b[i - 1] : 0.0;
        q = a[i] - x - (i ? off / q : 0.0);
        if (q == 0.0) q = -1e-300;
        if (q < 0) c++;
    }
    return c;
}

double lowest_eigenvalue(const std::vector<double>& a, const std::vector<double>& b, int m) {
    double lo = 1e300, hi = -1e300;  // Gershgorin bounds
    for (int i = 0; i < m; i++) {
        const double r = (i ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < m ? std::fabs(b[i]) : 0.0);
        lo = std::min(lo, a[i] - r);
        hi = std::max(hi, a[i] + r);
    }
    for (int it = 0; it < 200 && hi - lo > 1e-15 * std::max(1.0, std::fabs(lo) + std::fabs(hi)); it++) {
        const double mid = 0.5 * (lo + hi);
        if (sturm_count(a, b, m, mid) >= 1)
            hi = mid;
        else
            lo = mid;
    }
    return 0.5 * (lo + hi);
}

// eigenvector of the tridiagonal for eigenvalue lam: inverse iteration with
// the Thomas algorithm (a tiny shift keeps the factorisation regular)
std::vector<double> tridiag_vector(const std::vector<double>& a, const std::vector<double>& b, int m, double lam) {
    std::vector<double> x(m, 1.0), c(m), d(m), y(m);
    const double shift = lam - 1e-10 * std::max(1.0, std::fabs(lam));
    for (int pass = 0; pass < 3; pass++) {
        // solve (T - shift) y = x
        double den = a[0] - shift;
        if (den == 0) den = 1e-300;
        c[0] = m > 1 ? b[0] / den : 0.0;
        d[0] = x[0] / den;
        for (int i = 1; i < m; i++) {
            den = a[i] - shift - b[i - 1] * c[i - 1];
            if (den == 0) den = 1e-300;
            c[i] = i + 1 < m ? b[i] / den : 0.0;
            d[i] = (x[i] - b[i - 1] * d[i - 1]) / den;
        }
        y[m - 1] = d[m - 1];
        for (int i = m - 2; i >= 0; i--) y[i] = d[i] - c[i] * y[i + 1];
        double nrm = 0;
        for (int i = 0; i < m; i++) nrm += y[i] * y[i];
        nrm = std::sqrt(nrm);
        for (int i = 0; i < m; i++) x[i] = y[i] / nrm;
    }
    return x;
}

int grid_for(int64_t N) { return (int)std::min<int64_t>(kBlocks, std::max<int64_t>(1, (N + kThreads - 1) / kThreads)); }

}  // namespace

cudaError_t ed_ground_state(const HamDev& H, int n, int max_iter, double tol, uint64_t seed, cudaStream_t st,
                            double* energy, int* iterations, double2* psi_host) {
    const int64_t N = int64_t(1) << n;
    const int G = grid_for(N);
    double2 *v0 = nullptr, *v1 = nullptr, *w = nullptr, *part = nullptr, *sc = nullptr, *psi = nullptr;
    cudaError_t e = cudaSuccess;
    auto fail = [&](cudaError_t err) {
        cudaFree(v0);
        cudaFree(v1);
        cudaFree(w);
        cudaFree(part);
        cudaFree(sc);
        cudaFree(psi);
        return err;
    };
    if ((e = cudaMalloc(&v0, N * sizeof(double2))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&v1, N * sizeof(double2))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&w, N * sizeof(double2))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&part, kBlocks * sizeof(double2))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&sc, sizeof(double2))) != cudaSuccess) return fail(e);

    auto dot = [&](const double2* a, const double2* b, double2* out) -> cudaError_t {
        ed_dot<<<G, kThreads, 0, st>>>(a, b, N, part);
        ed_sum<<<1, 32, 0, st>>>(part, G, sc);
        cudaError_t err = cudaMemcpyAsync(out, sc, sizeof(double2), cudaMemcpyDeviceToHost, st);
        if (err != cudaSuccess) return err;
        return cudaStreamSynchronize(st);
    };
    // one Lanczos run; with coef, accumulate psi = sum_j coef[j] v_j
    std::vector<double> alpha, beta;
    auto run = [&](int m_max, const std::vector<double>* coef) -> cudaError_t {
        double2 nr;
        ed_start<<<G, kThreads, 0, st>>>(v0, N, seed);
        cudaError_t err = dot(v0, v0, &nr);
        if (err != cudaSuccess) return err;
        ed_scale<<<G, kThreads, 0, st>>>(v0, 1.0 / std::sqrt(nr.x), v0, N);
        double2* vp = nullptr;  // v_{j-1}
        double2* vc = v0;       // v_j
        double2* vn = v1;       // storage for v_{j+1}
        double bprev = 0.0, eprev = 0.0;
        int stable = 0;
        for (int j = 0; j < m_max; j++) {
            if (coef) ed_accumulate<<<G, kThreads, 0, st>>>(psi, vc, (*coef)[j], N);
            ed_apply<<<G, kThreads, 0, st>>>(H, N, vc, w);
            double2 aj;
            if ((err = dot(vc, w, &aj)) != cudaSuccess) return err;
            ed_axpy<<<G, kThreads, 0, st>>>(w, vc, vp, aj.x, bprev, N);
            double2 wn;
            if ((err = dot(w, w, &wn)) != cudaSuccess) return err;
            const double bj = std::sqrt(std::max(wn.x, 0.0));
            if (!coef) {
                alpha.push_back(aj.x);
                const int m = (int)alpha.size();
                const double ev = lowest_eigenvalue(alpha, beta, m);
                stable = (j > 0 && std::fabs(ev - eprev) <= tol * std::max(1.0, std::fabs(ev))) ? stable + 1 : 0;
                eprev = ev;
                if (stable >= 3 || bj <= 1e-12 * std::max(1.0, std::fabs(ev))) return cudaSuccess;
                beta.push_back(bj);
            } else if (j + 1 == m_max) {
                return cudaSuccess;
            }
            // v_{j+1} = w / b_j into the buffer of v_{j-1} (or v1 at the start)
            double2* dst = vp ? vp : vn;
            ed_scale<<<G, kThreads, 0, st>>>(w, 1.0 / (coef ? beta[j] : bj), dst, N);
            vp = vc;
            vc = dst;
            bprev = coef ? beta[j] : bj;
        }
        return cudaGetLastError();
    };
    if ((e = run(max_iter, nullptr)) != cudaSuccess) return fail(e);
    const int m = (int)alpha.size();
    const double ev = lowest_eigenvalue(alpha, beta, m);
    *energy = ev;
    if (iterations) *iterations = m;
    if (psi_host) {
        const std::vector<double> c = tridiag_vector(alpha, beta, m, ev);
        if ((e = cudaMalloc(&psi, N * sizeof(double2))) != cudaSuccess) return fail(e);
        if ((e = cudaMemsetAsync(psi, 0, N * sizeof(double2), st)) != cudaSuccess) return fail(e);
        if ((e = run(m, &c)) != cudaSuccess) return fail(e);
        double2 nr;
        if ((e = dot(psi, psi, &nr)) != cudaSuccess) return fail(e);
        ed_scale<<<G, kThreads, 0, st>>>(psi, 1.0 / std::sqrt(nr.x), psi, N);
        if ((e = cudaMemcpyAsync(psi_host, psi, N * sizeof(double2), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return fail(e);
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e);
    }
    return fail(cudaGetLastError());
}

}  // namespace rbmnqs
