// cosets.cu -- analysis of the symmetry group (host) and the kernels of the factorised symmetry
// transform / fold (device).  The algebra is stated in cosets.cuh.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <vector>

#include "cosets.cuh"

namespace tdscha {

// ================================================================================================
// Host analysis
// ================================================================================================
namespace {

// Eigen-decomposition of a symmetric d x d matrix (row-major) by cyclic Jacobi rotations:
// eigenvalues ascending in w, eigenvectors in the columns of V (row-major).
void jacobi_eigh(int d, std::vector<double> A, std::vector<double> &w, std::vector<double> &V) {
    V.assign((size_t)d * d, 0.0);
    for (int i = 0; i < d; ++i) V[(size_t)i * d + i] = 1.0;
    auto a = [&](int i, int j) -> double & { return A[(size_t)i * d + j]; };
    double scale = 0.0;
    for (double x : A) scale = std::max(scale, std::fabs(x));
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int i = 0; i < d; ++i)
            for (int j = i + 1; j < d; ++j) off = std::max(off, std::fabs(a(i, j)));
        if (off <= 1e-15 * std::max(scale, 1e-300)) break;
        for (int p = 0; p < d; ++p)
            for (int q = p + 1; q < d; ++q) {
                const double apq = a(p, q);
                if (std::fabs(apq) <= 1e-300) continue;
                const double theta = (a(q, q) - a(p, p)) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < d; ++k) {   // A <- J^T A J on columns p, q
                    const double akp = a(k, p), akq = a(k, q);
                    a(k, p) = c * akp - s * akq;
                    a(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < d; ++k) {   // rows p, q
                    const double apk = a(p, k), aqk = a(q, k);
                    a(p, k) = c * apk - s * aqk;
                    a(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < d; ++k) {
                    const double vkp = V[(size_t)k * d + p], vkq = V[(size_t)k * d + q];
                    V[(size_t)k * d + p] = c * vkp - s * vkq;
                    V[(size_t)k * d + q] = s * vkp + c * vkq;
                }
            }
    }
    std::vector<int> idx(d);
    for (int i = 0; i < d; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int x, int y) { return a(x, x) < a(y, y); });
    w.resize(d);
    std::vector<double> Vs((size_t)d * d);
    for (int c = 0; c < d; ++c) {
        w[c] = a(idx[c], idx[c]);
        for (int k = 0; k < d; ++k) Vs[(size_t)k * d + c] = V[(size_t)k * d + idx[c]];
    }
    V.swap(Vs);
}

// deterministic weights in [0.5, 1.5) for the random combinations of the subgroup's matrices
double weight(uint64_t &s) {
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    return 0.5 + (double)(s >> 11) * (1.0 / 9007199254740992.0);
}

// Rotation R (d x d) of one block that brings every matrix of the subgroup (mats: |K| tables of
// d x d) to 1 x 1 / 2 x 2 blocks; partner (local indices).  Returns false when the subgroup's
// representation on the block has an isotypic component that is neither real (all +-1) nor a
// complex pair (for an abelian subgroup it always is one or the other).
bool block_rotation(int d, const std::vector<const double *> &mats, std::vector<double> &R, std::vector<int> &partner) {
    const size_t dd = (size_t)d * d;
    std::vector<double> Msym(dd, 0.0), Manti(dd, 0.0);
    uint64_t seed = 0x9E3779B97F4A7C15ULL;
    for (const double *M : mats) {
        const double c = weight(seed), c2 = weight(seed);
        for (int i = 0; i < d; ++i)
            for (int j = 0; j < d; ++j) {
                Msym[(size_t)i * d + j] += c * (M[(size_t)i * d + j] + M[(size_t)j * d + i]);
                Manti[(size_t)i * d + j] += c2 * (M[(size_t)i * d + j] - M[(size_t)j * d + i]);
            }
    }
    std::vector<double> lam, Q;
    jacobi_eigh(d, Msym, lam, Q);
    double lmax = 1.0;
    for (double x : lam) lmax = std::max(lmax, std::fabs(x));
    // clusters of equal eigenvalue = isotypic components (a real character, or a complex pair)
    std::vector<std::pair<int, int>> cl;   // [begin, end)
    int b = 0;
    for (int i = 1; i <= d; ++i)
        if (i == d || std::fabs(lam[i] - lam[i - 1]) > 1e-6 * lmax) { cl.push_back({b, i}); b = i; }
    R.assign(dd, 0.0);
    partner.assign(d, 0);
    int col = 0;
    const double kscale = (double)mats.size() * (double)mats.size();
    for (auto [c0, c1] : cl) {
        const int m = c1 - c0;
        // A = Qc^T Manti Qc (m x m)
        std::vector<double> T((size_t)d * m, 0.0), A((size_t)m * m, 0.0);
        for (int i = 0; i < d; ++i)
            for (int q = 0; q < m; ++q) {
                double s = 0.0;
                for (int k = 0; k < d; ++k) s += Manti[(size_t)i * d + k] * Q[(size_t)k * d + c0 + q];
                T[(size_t)i * m + q] = s;
            }
        double a2 = 0.0;
        for (int p = 0; p < m; ++p)
            for (int q = 0; q < m; ++q) {
                double s = 0.0;
                for (int i = 0; i < d; ++i) s += Q[(size_t)i * d + c0 + p] * T[(size_t)i * m + q];
                A[(size_t)p * m + q] = s;
                a2 += s * s;
            }
        a2 /= m;   // -trace(A A) / m
        std::vector<std::vector<double>> loc;   // basis of the cluster in its own coordinates
        std::vector<int> lpart;
        if (a2 < 1e-14 * kscale) {              // real character: every matrix is +-1 here
            for (int q = 0; q < m; ++q) {
                std::vector<double> v(m, 0.0);
                v[q] = 1.0;
                loc.push_back(v);
                lpart.push_back(q);
            }
        } else {                                // complex pair: every matrix is cos I + sin J here
            if (m % 2) return false;
            const double inv = 1.0 / std::sqrt(a2);
            for (int q = 0; q < m && (int)loc.size() < m; ++q) {
                std::vector<double> v(m, 0.0);
                v[q] = 1.0;
                for (const auto &u : loc) {
                    double dot = 0.0;
                    for (int i = 0; i < m; ++i) dot += u[i] * v[i];
                    for (int i = 0; i < m; ++i) v[i] -= dot * u[i];
                }
                double nv = 0.0;
                for (double x : v) nv += x * x;
                if (nv < 1e-6) continue;
                nv = 1.0 / std::sqrt(nv);
                for (double &x : v) x *= nv;
                std::vector<double> w(m, 0.0);   // J v
                for (int i = 0; i < m; ++i) {
                    double s = 0.0;
                    for (int k = 0; k < m; ++k) s += A[(size_t)i * m + k] * v[k];
                    w[i] = s * inv;
                }
                double nw = 0.0;
                for (double x : w) nw += x * x;
                if (nw < 0.25) return false;
                nw = 1.0 / std::sqrt(nw);
                for (double &x : w) x *= nw;
                const int k0 = (int)loc.size();
                loc.push_back(v);
                loc.push_back(w);
                lpart.push_back(k0 + 1);
                lpart.push_back(k0);
            }
            if ((int)loc.size() != m) return false;
        }
        for (int q = 0; q < m; ++q) {
            for (int i = 0; i < d; ++i) {
                double s = 0.0;
                for (int k = 0; k < m; ++k) s += Q[(size_t)i * d + c0 + k] * loc[q][k];
                R[(size_t)i * d + col + q] = s;
            }
            partner[col + q] = col + lpart[q];
        }
        col += m;
    }
    // orthonormality
    for (int p = 0; p < d; ++p)
        for (int q = 0; q < d; ++q) {
            double s = 0.0;
            for (int i = 0; i < d; ++i) s += R[(size_t)i * d + p] * R[(size_t)i * d + q];
            if (std::fabs(s - (p == q ? 1.0 : 0.0)) > 1e-10) return false;
        }
    return true;
}

// largest |(R^T M R)[x][q]| outside x in {q, pi(q)}
double offpattern_of(int d, const double *M, const std::vector<double> &R, const std::vector<int> &partner) {
    std::vector<double> T((size_t)d * d, 0.0);
    for (int i = 0; i < d; ++i)
        for (int q = 0; q < d; ++q) {
            double s = 0.0;
            for (int k = 0; k < d; ++k) s += M[(size_t)i * d + k] * R[(size_t)k * d + q];
            T[(size_t)i * d + q] = s;
        }
    double off = 0.0;
    for (int x = 0; x < d; ++x)
        for (int q = 0; q < d; ++q) {
            if (x == q || x == partner[q]) continue;
            double s = 0.0;
            for (int i = 0; i < d; ++i) s += R[(size_t)i * d + x] * T[(size_t)i * d + q];
            off = std::max(off, std::fabs(s));
        }
    return off;
}

}  // namespace

int analyse_cosets(int N_sym, const std::vector<int> &dim, const double *const *sym_blocks, CosetAnalysis &out) {
    out = CosetAnalysis();
    const int nblk = (int)dim.size();
    int n = 0;
    for (int d : dim) n += d;
    // kernel of every block's representation
    std::vector<std::vector<int>> kern(nblk);
    for (int b = 0; b < nblk; ++b) {
        const int d = dim[b];
        for (int j = 0; j < N_sym; ++j) {
            const double *M = sym_blocks[b] + (size_t)j * d * d;
            double dev = 0.0;
            for (int p = 0; p < d && dev < 1e-6; ++p)
                for (int q = 0; q < d; ++q) dev = std::max(dev, std::fabs(M[(size_t)p * d + q] - (p == q ? 1.0 : 0.0)));
            if (dev < 1e-6) kern[b].push_back(j);
        }
    }
    std::vector<int> cand(nblk);
    for (int b = 0; b < nblk; ++b) cand[b] = b;
    std::stable_sort(cand.begin(), cand.end(), [&](int x, int y) { return kern[x].size() > kern[y].size(); });
    out.why = "no block whose representation has a proper kernel of order >= 4";
    std::vector<std::vector<int>> tried;
    for (int b0 : cand) {
        const auto &K = kern[b0];
        const int sub = (int)K.size();
        if (sub < 4 || sub >= N_sym || N_sym % sub) continue;
        if (std::find(tried.begin(), tried.end(), K) != tried.end()) continue;
        tried.push_back(K);
        if (tried.size() > 3) break;
        // rotation of every block from the subgroup's matrices
        std::vector<double> R;
        std::vector<long long> R_off(nblk);
        std::vector<int> partner(n);
        bool ok = true;
        double off = 0.0;
        int s = 0;
        for (int b = 0; b < nblk && ok; ++b) {
            const int d = dim[b];
            std::vector<const double *> mats;
            for (int j : K) mats.push_back(sym_blocks[b] + (size_t)j * d * d);
            std::vector<double> Rb;
            std::vector<int> pb;
            if (!block_rotation(d, mats, Rb, pb)) { ok = false; out.why = "subgroup not reducible to 2 x 2 blocks"; break; }
            for (const double *M : mats) off = std::max(off, offpattern_of(d, M, Rb, pb));
            R_off[b] = (long long)R.size();
            R.insert(R.end(), Rb.begin(), Rb.end());
            for (int q = 0; q < d; ++q) partner[s + q] = s + pb[q];
            s += d;
        }
        if (!ok) continue;
        if (off > 1e-7) { out.why = "subgroup matrices not 2 x 2 sparse in the rotated basis"; continue; }
        // cosets = classes of equal S_j on block b0
        const int d0 = dim[b0];
        std::map<std::vector<long long>, int> key_of;
        std::vector<std::vector<int>> members;
        for (int j = 0; j < N_sym; ++j) {
            const double *M = sym_blocks[b0] + (size_t)j * d0 * d0;
            std::vector<long long> key((size_t)d0 * d0);
            for (int i = 0; i < d0 * d0; ++i) key[i] = std::llround(M[i] * 1e6);
            auto it = key_of.find(key);
            if (it == key_of.end()) {
                key_of.emplace(key, (int)members.size());
                members.push_back({j});
            } else {
                members[it->second].push_back(j);
            }
        }
        bool uniform = true;
        for (const auto &m : members) uniform = uniform && (int)m.size() == sub;
        if (!uniform) { out.why = "cosets of unequal size"; continue; }
        out.ok = true;
        out.b0 = b0;
        out.sub = sub;
        out.n_cos = (int)members.size();
        out.kset = K;
        out.order.clear();
        for (const auto &m : members) out.order.insert(out.order.end(), m.begin(), m.end());
        out.partner = partner;
        out.R = R;
        out.R_off = R_off;
        out.offpattern = off;
        out.why.clear();
        return 0;
    }
    return 0;
}

// ================================================================================================
// Device kernels
// ================================================================================================
namespace {

__device__ __forceinline__ long long packed(int a, int b, int n) {   // packed index of (min, max)
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    return (long long)lo * n - ((long long)lo * (lo - 1)) / 2 + (hi - lo);
}

// every row of an (rows x n) array: to_rot out[s+q] = sum_q' R_b[q'][q] in[s+q'], else
// out[s+q'] = sum_q R_b[q'][q] in[s+q]
__global__ void rotate_rows_kernel(long long rows, int n, int dmax, const double *__restrict__ Rrow,
                                   const int *__restrict__ blocks_ids, const int *__restrict__ blk_start,
                                   const int *__restrict__ blk_dim, const double *__restrict__ in, double *__restrict__ out,
                                   bool to_rot) {
    const long long total = rows * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const long long r = idx / n;
        const int x = (int)(idx - r * n);
        const int b = blocks_ids[x], s = blk_start[b], d = blk_dim[b];
        const double *v = in + r * n + s;
        double acc = 0.0;
        if (to_rot)
            for (int y = 0; y < d; ++y) acc += Rrow[(long long)(s + y) * dmax + (x - s)] * v[y];
        else
            for (int y = 0; y < d; ++y) acc += Rrow[(long long)x * dmax + y] * v[y];
        out[idx] = acc;
    }
}

// the row index of each (n x n) matrix: to_rot out[s+q][c] = sum_q' R_b[q'][q] in[s+q'][c], else
// out[s+q'][c] = sum_q R_b[q'][q] in[s+q][c]
__global__ void rotate_cols_kernel(int nb, int n, int dmax, const double *__restrict__ Rrow, const int *__restrict__ blocks_ids,
                                   const int *__restrict__ blk_start, const int *__restrict__ blk_dim,
                                   const double *__restrict__ in, double *__restrict__ out, bool to_rot) {
    const long long nn = (long long)n * n, total = (long long)nb * nn;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const long long k = idx / nn;
        const long long e = idx - k * nn;
        const int x = (int)(e / n), c = (int)(e - (long long)x * n);
        const int b = blocks_ids[x], s = blk_start[b], d = blk_dim[b];
        const double *A = in + k * nn + c;
        double acc = 0.0;
        if (to_rot)
            for (int y = 0; y < d; ++y) acc += Rrow[(long long)(s + y) * dmax + (x - s)] * A[(long long)(s + y) * n];
        else
            for (int y = 0; y < d; ++y) acc += Rrow[(long long)x * dmax + y] * A[(long long)(s + y) * n];
        out[idx] = acc;
    }
}

// M' = R^T M R for the tables of one block, one CTA per symmetry
__global__ void rotate_tables_kernel(double *__restrict__ sym, int d, const double *__restrict__ Rb) {
    extern __shared__ double sh[];
    double *Rs = sh, *Ms = sh + d * d, *Ts = sh + 2 * d * d;
    double *M = sym + (long long)blockIdx.x * d * d;
    for (int i = threadIdx.x; i < d * d; i += blockDim.x) { Rs[i] = Rb[i]; Ms[i] = M[i]; }
    __syncthreads();
    for (int i = threadIdx.x; i < d * d; i += blockDim.x) {   // T = M R
        const int p = i / d, q = i - p * d;
        double s = 0.0;
        for (int k = 0; k < d; ++k) s += Ms[p * d + k] * Rs[k * d + q];
        Ts[i] = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < d * d; i += blockDim.x) {   // M' = R^T T
        const int p = i / d, q = i - p * d;
        double s = 0.0;
        for (int k = 0; k < d; ++k) s += Rs[k * d + p] * Ts[k * d + q];
        M[i] = s;
    }
}

// c0 / c1 of D_j = S_p^T S_j (rotated tables) per (internal row, mode); the largest entry outside
// the pattern goes to offmax
__global__ void coset_coef_kernel(int N_sym, int n, int sub, const int *__restrict__ order, const int *__restrict__ partner,
                                  const int *__restrict__ blocks_ids, const int *__restrict__ blk_start,
                                  const int *__restrict__ blk_dim, const double *__restrict__ sym,
                                  const long long *__restrict__ blk_sym_off, float *__restrict__ c0, float *__restrict__ c1,
                                  unsigned long long *offmax) {
    const long long total = (long long)N_sym * n;
    double off = 0.0;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const int jr = (int)(idx / n), mu = (int)(idx - (long long)jr * n);
        const int j = order[jr], p = order[(jr / sub) * sub];
        const int b = blocks_ids[mu], s = blk_start[b], d = blk_dim[b];
        const int q = mu - s, pq = partner[mu] - s;
        const double *Mp = sym + blk_sym_off[b] + (long long)p * d * d;
        const double *Mj = sym + blk_sym_off[b] + (long long)j * d * d;
        double v0 = 0.0, v1 = 0.0;
        for (int x = 0; x < d; ++x) {
            double acc = 0.0;
            for (int a = 0; a < d; ++a) acc += Mp[a * d + x] * Mj[a * d + q];
            if (x == q) v0 = acc;
            else if (x == pq) v1 = acc;
            else off = fmax(off, fabs(acc));
        }
        c0[idx] = (float)v0;
        c1[idx] = pq != q ? (float)v1 : 0.f;
    }
    // non-negative doubles order like their bit patterns
    atomicMax(offmax, (unsigned long long)__double_as_longlong(off));
}

// B1 expansion: one CTA per (4 x 256 packed pairs, coset row); loops over the coset's rows
template <Format FMT>
__global__ void __launch_bounds__(256) coset_expand_kernel(int ncj, int sub, int j0, long long P, long long Kp, int n,
                                                           const float *__restrict__ U, const int *__restrict__ pmu,
                                                           const int *__restrict__ pnu, const int *__restrict__ partner,
                                                           const float *__restrict__ c0, const float *__restrict__ c1,
                                                           void *B1_hi, void *B1_lo) {
    const long long urow = blockIdx.y;
    const int k = (int)(urow / ncj), pc = (int)(urow - (long long)k * ncj);
    const long long nj = (long long)ncj * sub;
    const long long p0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 4;
    if (p0 >= Kp) return;
    const float *Ur = U + urow * Kp;
    float u[4][4];
    int mu[4], nu[4];
    bool valid[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const long long p = p0 + e;
        valid[e] = p < P;
        mu[e] = valid[e] ? pmu[p] : 0;
        nu[e] = valid[e] ? pnu[p] : 0;
        if (valid[e]) {
            const int pm = partner[mu[e]], pn = partner[nu[e]];
            u[e][0] = Ur[packed(mu[e], nu[e], n)];
            u[e][1] = Ur[packed(mu[e], pn, n)];
            u[e][2] = Ur[packed(pm, nu[e], n)];
            u[e][3] = Ur[packed(pm, pn, n)];
        } else {
            u[e][0] = u[e][1] = u[e][2] = u[e][3] = 0.f;
        }
    }
    const bool lo = B1_lo != nullptr;
    for (int t = 0; t < sub; ++t) {
        const long long jr = (long long)j0 + (long long)pc * sub + t;
        const long long r = (long long)k * nj + (long long)pc * sub + t;
        const float *C0 = c0 + jr * n, *C1 = c1 + jr * n;
        float x[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            if (valid[e]) {
                const float a0 = C0[mu[e]], a1 = C1[mu[e]], b0 = C0[nu[e]], b1 = C1[nu[e]];
                x[e] = a0 * (b0 * u[e][0] + b1 * u[e][1]) + a1 * (b0 * u[e][2] + b1 * u[e][3]);
            } else {
                x[e] = 0.f;
            }
        }
        const long long o = r * Kp + p0;
        if constexpr (FMT == FMT_BF16) {
            __nv_bfloat16 h[4], l[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                h[e] = __float2bfloat16_rn(x[e]);
                l[e] = __float2bfloat16_rn(x[e] - __bfloat162float(h[e]));
            }
            *reinterpret_cast<uint2 *>(static_cast<__nv_bfloat16 *>(B1_hi) + o) = *reinterpret_cast<const uint2 *>(h);
            if (lo) *reinterpret_cast<uint2 *>(static_cast<__nv_bfloat16 *>(B1_lo) + o) = *reinterpret_cast<const uint2 *>(l);
        } else {
            float4 h, l;
            h.x = tf32_round(x[0]); h.y = tf32_round(x[1]); h.z = tf32_round(x[2]); h.w = tf32_round(x[3]);
            l.x = tf32_round(x[0] - h.x); l.y = tf32_round(x[1] - h.y); l.z = tf32_round(x[2] - h.z); l.w = tf32_round(x[3] - h.w);
            *reinterpret_cast<float4 *>(static_cast<float *>(B1_hi) + o) = h;
            if (lo) *reinterpret_cast<float4 *>(static_cast<float *>(B1_lo) + o) = l;
        }
    }
}

__global__ void coset_expand_r1_kernel(int nb, int ncj, int sub, int j0, int n, long long np, const float *__restrict__ r1p,
                                       const int *__restrict__ partner, const float *__restrict__ c0,
                                       const float *__restrict__ c1, Format fmt, void *r1_hi, void *r1_lo) {
    const long long nj = (long long)ncj * sub, total = (long long)nb * nj * np;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const long long r = idx / np;
        const int mu = (int)(idx - r * np);
        const long long k = r / nj, l = r - k * nj;
        double v = 0.0;
        if (mu < n) {
            const long long jr = j0 + l;
            const float *src = r1p + (k * ncj + l / sub) * np;
            v = (double)(c0[jr * n + mu] * src[mu] + c1[jr * n + mu] * src[partner[mu]]);
        }
        store_split(fmt, r1_hi, r1_lo, idx, v);
    }
}

// fold, inner part: one CTA per (256 packed pairs, coset row); FP64 sums over the coset's rows
__global__ void __launch_bounds__(256) coset_fold_inner_kernel(int ncj, int sub, int j0, long long P, long long ldz, int n,
                                                               const float *__restrict__ Z, const int *__restrict__ pmu,
                                                               const int *__restrict__ pnu, const int *__restrict__ partner,
                                                               const float *__restrict__ c0, const float *__restrict__ c1,
                                                               float *__restrict__ Zs) {
    const long long urow = blockIdx.y;
    const int k = (int)(urow / ncj), pc = (int)(urow - (long long)k * ncj);
    const long long nj = (long long)ncj * sub;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const int a = pmu[p], b = pnu[p], pa = partner[a], pb = partner[b];
    const long long i00 = packed(a, b, n), i01 = packed(a, pb, n), i10 = packed(pa, b, n), i11 = packed(pa, pb, n);
    const float e00 = a == b ? 2.f : 1.f, e01 = a == pb ? 2.f : 1.f, e10 = pa == b ? 2.f : 1.f, e11 = pa == pb ? 2.f : 1.f;
    const bool ha = pa != a, hb = pb != b;
    double acc = 0.0;
    for (int t = 0; t < sub; ++t) {
        const long long jr = (long long)j0 + (long long)pc * sub + t;
        const float *Zr = Z + ((long long)k * nj + (long long)pc * sub + t) * ldz;
        const float *C0 = c0 + jr * n, *C1 = c1 + jr * n;
        const float A0 = C0[a], A1 = ha ? C1[pa] : 0.f, B0 = C0[b], B1 = hb ? C1[pb] : 0.f;
        const float z00 = e00 * Zr[i00], z01 = e01 * Zr[i01], z10 = e10 * Zr[i10], z11 = e11 * Zr[i11];
        acc += (double)(A0 * (B0 * z00 + B1 * z01)) + (double)(A1 * (B0 * z10 + B1 * z11));
    }
    Zs[urow * ldz + p] = (float)(acc / (double)e00);
}

__global__ void coset_fold_inner_f_kernel(int nb, int ncj, int sub, int j0, long long ldf, int n, const float *__restrict__ F,
                                          const int *__restrict__ partner, const float *__restrict__ c0,
                                          const float *__restrict__ c1, float *__restrict__ Fs) {
    const long long nj = (long long)ncj * sub, total = (long long)nb * ncj * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const long long urow = idx / n;
        const int a = (int)(idx - urow * n), pa = partner[a];
        const long long k = urow / ncj, pc = urow - k * ncj;
        double acc = 0.0;
        for (int t = 0; t < sub; ++t) {
            const long long jr = j0 + pc * sub + t;
            const float *Fr = F + (k * nj + pc * sub + t) * ldf;
            acc += (double)c0[jr * n + a] * Fr[a];
            if (pa != a) acc += (double)c1[jr * n + pa] * Fr[pa];
        }
        Fs[urow * ldf + a] = (float)acc;
    }
}

inline unsigned grid_of(long long work) { return (unsigned)std::min<long long>((work + 255) / 256, 148LL * 32); }

}  // namespace

int rotate_rows_of(long long rows, int n, int dmax, const double *Rrow, const int *blocks_ids, const int *blk_start,
                   const int *blk_dim, const double *in, double *out, bool to_rot, cudaStream_t st) {
    if (rows <= 0) return 0;
    rotate_rows_kernel<<<grid_of(rows * n), 256, 0, st>>>(rows, n, dmax, Rrow, blocks_ids, blk_start, blk_dim, in, out, to_rot);
    TD_CUDA(cudaGetLastError());
    return 0;
}

int rotate_mats(int nb, int n, int dmax, const double *Rrow, const int *blocks_ids, const int *blk_start, const int *blk_dim,
                const double *in, double *tmp, double *out, bool to_rot, cudaStream_t st) {
    // column index first (every row of every matrix), then the row index
    TD_TRY(rotate_rows_of((long long)nb * n, n, dmax, Rrow, blocks_ids, blk_start, blk_dim, in, tmp, to_rot, st));
    rotate_cols_kernel<<<grid_of((long long)nb * n * n), 256, 0, st>>>(nb, n, dmax, Rrow, blocks_ids, blk_start, blk_dim, tmp, out,
                                                                       to_rot);
    TD_CUDA(cudaGetLastError());
    return 0;
}

int rotate_sym_tables(double *sym_b, int N_sym, int d, const double *Rb, cudaStream_t st) {
    const size_t smem = (size_t)3 * d * d * sizeof(double);
    TD_CUDA(cudaFuncSetAttribute(rotate_tables_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    rotate_tables_kernel<<<N_sym, 256, smem, st>>>(sym_b, d, Rb);
    TD_CUDA(cudaGetLastError());
    return 0;
}

int coset_coefficients(int N_sym, int n, int sub, const int *order, const int *partner, const int *blocks_ids,
                       const int *blk_start, const int *blk_dim, const double *sym, const long long *blk_sym_off, float *c0,
                       float *c1, unsigned long long *offmax, cudaStream_t st) {
    coset_coef_kernel<<<grid_of((long long)N_sym * n), 256, 0, st>>>(N_sym, n, sub, order, partner, blocks_ids, blk_start,
                                                                     blk_dim, sym, blk_sym_off, c0, c1, offmax);
    TD_CUDA(cudaGetLastError());
    return 0;
}

int coset_expand(int nb, int ncj, int sub, int j0, long long P, long long Kp, int n, const float *U, const int *pmu,
                 const int *pnu, const int *partner, const float *c0, const float *c1, Format fmt, void *B1_hi, void *B1_lo,
                 cudaStream_t st) {
    TD_CHECK(Kp % 4 == 0, TDSCHA_EINVAL, "packed row length %lld is not a multiple of 4", Kp);
    TD_CHECK((long long)nb * ncj <= 65535, TDSCHA_EINVAL, "%d coset rows exceed the expansion grid", nb * ncj);
    dim3 grid((unsigned)ceil_div(Kp, 1024), (unsigned)(nb * ncj));
    if (fmt == FMT_BF16)
        coset_expand_kernel<FMT_BF16><<<grid, 256, 0, st>>>(ncj, sub, j0, P, Kp, n, U, pmu, pnu, partner, c0, c1, B1_hi, B1_lo);
    else if (fmt == FMT_TF32)
        coset_expand_kernel<FMT_TF32><<<grid, 256, 0, st>>>(ncj, sub, j0, P, Kp, n, U, pmu, pnu, partner, c0, c1, B1_hi, B1_lo);
    else
        TD_CHECK(false, TDSCHA_EINVAL, "coset expansion needs a split storage format");
    TD_CUDA(cudaGetLastError());
    return 0;
}

int coset_expand_r1(int nb, int ncj, int sub, int j0, int n, long long np, const float *r1p, const int *partner,
                    const float *c0, const float *c1, Format fmt, void *r1_hi, void *r1_lo, cudaStream_t st) {
    coset_expand_r1_kernel<<<grid_of((long long)nb * ncj * sub * np), 256, 0, st>>>(nb, ncj, sub, j0, n, np, r1p, partner, c0,
                                                                                      c1, fmt, r1_hi, r1_lo);
    TD_CUDA(cudaGetLastError());
    return 0;
}

int coset_fold_inner(int nb, int ncj, int sub, int j0, long long P, long long ldz, long long ldf, int n, const float *Z,
                     const float *F, const int *pmu, const int *pnu, const int *partner, const float *c0, const float *c1,
                     float *Zs, float *Fs, cudaStream_t st) {
    TD_CHECK((long long)nb * ncj <= 65535, TDSCHA_EINVAL, "%d coset rows exceed the fold grid", nb * ncj);
    dim3 grid((unsigned)ceil_div(P, 256), (unsigned)(nb * ncj));
    coset_fold_inner_kernel<<<grid, 256, 0, st>>>(ncj, sub, j0, P, ldz, n, Z, pmu, pnu, partner, c0, c1, Zs);
    coset_fold_inner_f_kernel<<<grid_of((long long)nb * ncj * n), 256, 0, st>>>(nb, ncj, sub, j0, ldf, n, F, partner, c0, c1, Fs);
    TD_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace tdscha
