// freq.cu -- character classes of the symmetry subgroup (host) and the operand / left-operand /
// reconstruction kernels of the averages in the character basis (device).  The algebra is stated in
// freq.cuh.
#include <algorithm>
#include <cmath>
#include <complex>
#include <map>
#include <vector>

#include "freq.cuh"

namespace tdscha {

// ================================================================================================
// Host: classes and layouts
// ================================================================================================
namespace {

using Chi = std::vector<std::complex<double>>;

std::vector<long long> chi_key(const Chi &c, bool conj) {
    std::vector<long long> k(2 * c.size());
    for (size_t t = 0; t < c.size(); ++t) {
        k[2 * t] = std::llround(c[t].real() * 1e6);
        k[2 * t + 1] = std::llround((conj ? -c[t].imag() : c[t].imag()) * 1e6);
    }
    return k;
}

Chi chi_mul(const Chi &a, const Chi &b, bool conj_b) {
    Chi r(a.size());
    for (size_t t = 0; t < a.size(); ++t) r[t] = a[t] * (conj_b ? std::conj(b[t]) : b[t]);
    return r;
}

struct Term {
    int mu, nu;
    double c;
};

// One component of the symmetric-matrix space: real part = sum re, imaginary part = sum im of the
// matrix entries (im empty for a real scalar component), character chi, Frobenius multiplicity m.
struct Comp {
    int cls = -1;
    bool conj = false;
    double m = 1;
    std::vector<Term> re, im;
    int col = -1;   // first column (the imaginary part is at col + 1)
};

// M[mu, nu] += c * (part 0: real, 1: imaginary) of component k
struct Recon {
    int mu, nu, comp, part;
    double c;
};

}  // namespace

int build_freq_layout(int n, const std::vector<int> &dim, const std::vector<int> &blk_start, const double *const *sym_blocks,
                      const CosetAnalysis &ca, FreqLayout &out) {
    out = FreqLayout();
    if (!ca.ok || (int)ca.kset.size() != ca.sub) return 0;
    const int sub = ca.sub;
    const int nblk = (int)dim.size();
    // characters of every rotated mode on the subgroup: chi_q(t) = D_t[q, q] + i D_t[pi(q), q]
    std::vector<Chi> chi(n, Chi(sub));
    for (int b = 0; b < nblk; ++b) {
        const int d = dim[b], s = blk_start[b];
        const double *R = ca.R.data() + ca.R_off[b];
        std::vector<double> T((size_t)d * d);
        for (int t = 0; t < sub; ++t) {
            const double *S = sym_blocks[b] + (size_t)ca.kset[t] * d * d;
            for (int k = 0; k < d; ++k)
                for (int q = 0; q < d; ++q) {
                    double acc = 0.0;
                    for (int l = 0; l < d; ++l) acc += S[(size_t)k * d + l] * R[(size_t)l * d + q];
                    T[(size_t)k * d + q] = acc;
                }
            for (int q = 0; q < d; ++q) {
                const int pq = ca.partner[s + q] - s;
                double re = 0.0, im = 0.0;
                for (int k = 0; k < d; ++k) re += R[(size_t)k * d + q] * T[(size_t)k * d + q];
                if (pq != q)
                    for (int k = 0; k < d; ++k) im += R[(size_t)k * d + pq] * T[(size_t)k * d + q];
                chi[s + q][t] = {re, im};
            }
        }
    }
    std::map<std::vector<long long>, int> cls_of;
    std::vector<int> cls_real;
    auto classify = [&](const Chi &c, bool &conj) {
        const auto kc = chi_key(c, false), kb = chi_key(c, true);
        const bool real = kc == kb;
        conj = !real && kb < kc;
        const auto &canon = conj ? kb : kc;
        auto it = cls_of.find(canon);
        if (it != cls_of.end()) return it->second;
        const int id = (int)cls_real.size();
        cls_of.emplace(canon, id);
        cls_real.push_back(real ? 1 : 0);
        return id;
    };
    // orbits: a real mode, or a complex pair (lead, partner) with lead < partner
    std::vector<std::pair<int, int>> orbits;
    for (int q = 0; q < n; ++q) {
        const int pq = ca.partner[q];
        if (pq == q) orbits.push_back({q, -1});
        else if (q < pq) orbits.push_back({q, pq});
    }
    // pair components and the reconstruction of every matrix entry from them
    std::vector<Comp> comps;
    std::vector<Recon> recon;
    const Chi one(sub, {1.0, 0.0});
    auto add = [&](const Chi &c, double m, std::vector<Term> re, std::vector<Term> im) {
        Comp k;
        k.cls = classify(c, k.conj);
        k.m = m;
        k.re = std::move(re);
        k.im = std::move(im);
        comps.push_back(std::move(k));
        return (int)comps.size() - 1;
    };
    const int no = (int)orbits.size();
    for (int a = 0; a < no; ++a)
        for (int b = a; b < no; ++b) {
            int q = orbits[a].first, qb = orbits[a].second, r = orbits[b].first, rb = orbits[b].second;
            if (qb >= 0 && rb >= 0 && a != b) {
                // 2 x 2 block: linear part (chi_q conj chi_r) and antilinear part (chi_q chi_r)
                const int L = add(chi_mul(chi[q], chi[r], true), 4.0, {{q, r, 0.5}, {qb, rb, 0.5}}, {{qb, r, 0.5}, {q, rb, -0.5}});
                const int A = add(chi_mul(chi[q], chi[r], false), 4.0, {{q, r, 0.5}, {qb, rb, -0.5}}, {{q, rb, 0.5}, {qb, r, 0.5}});
                recon.push_back({q, r, L, 0, 1.0}); recon.push_back({q, r, A, 0, 1.0});
                recon.push_back({qb, rb, L, 0, 1.0}); recon.push_back({qb, rb, A, 0, -1.0});
                recon.push_back({qb, r, L, 1, 1.0}); recon.push_back({qb, r, A, 1, 1.0});
                recon.push_back({q, rb, L, 1, -1.0}); recon.push_back({q, rb, A, 1, 1.0});
            } else if (qb >= 0 && a == b) {
                // diagonal 2 x 2 block: trace part (trivial character) and antilinear part (chi_q^2)
                const int L = add(one, 2.0, {{q, q, 0.5}, {qb, qb, 0.5}}, {});
                const int A = add(chi_mul(chi[q], chi[q], false), 2.0, {{q, q, 0.5}, {qb, qb, -0.5}}, {{q, qb, 1.0}});
                recon.push_back({q, q, L, 0, 1.0}); recon.push_back({q, q, A, 0, 1.0});
                recon.push_back({qb, qb, L, 0, 1.0}); recon.push_back({qb, qb, A, 0, -1.0});
                recon.push_back({q, qb, A, 1, 1.0});
            } else if (qb >= 0 || rb >= 0) {
                if (qb >= 0) { std::swap(q, r); std::swap(qb, rb); }   // q real, (r, rb) complex
                const int W = add(chi_mul(chi[q], chi[r], false), 2.0, {{q, r, 1.0}}, {{q, rb, 1.0}});
                recon.push_back({q, r, W, 0, 1.0});
                recon.push_back({q, rb, W, 1, 1.0});
            } else {
                const int S = add(chi_mul(chi[q], chi[r], false), q == r ? 1.0 : 2.0, {{q, r, 1.0}}, {});
                recon.push_back({q, r, S, 0, 1.0});
            }
        }
    const long long P = (long long)n * (n + 1) / 2;
    // mode components (orbits) and their classes
    struct ModeComp {
        int cls;
        bool conj;
        int q, qb;
        int col;
    };
    std::vector<ModeComp> mcomps;
    for (auto [q, qb] : orbits) {
        ModeComp mc{};
        mc.cls = classify(chi[q], mc.conj);
        mc.q = q;
        mc.qb = qb;
        mcomps.push_back(mc);
    }
    const int ncls = (int)cls_real.size();
    std::vector<std::vector<int>> by_cls(ncls), mby_cls(ncls);
    for (int k = 0; k < (int)comps.size(); ++k) by_cls[comps[k].cls].push_back(k);
    for (int k = 0; k < (int)mcomps.size(); ++k) mby_cls[mcomps[k].cls].push_back(k);
    // column layout, class by class (classes without pair components drop out: they carry nothing)
    int kq = 0, kmq = 0;
    std::vector<int> keep;
    for (int g = 0; g < ncls; ++g) {
        if (by_cls[g].empty()) continue;
        const int id = (int)keep.size();
        keep.push_back(g);
        out.cls_real.push_back(cls_real[g]);
        out.pcol_off.push_back(kq);
        int cnt = 0;
        for (int k : by_cls[g]) { comps[k].col = kq + cnt; cnt += comps[k].im.empty() ? 1 : 2; }
        out.pcol_cnt.push_back((int)round_up(cnt, 64));
        kq += out.pcol_cnt.back();
        out.mcol_off.push_back(kmq);
        int mcnt = 0;
        for (int k : mby_cls[g]) { mcomps[k].col = kmq + mcnt; mcnt += mcomps[k].qb >= 0 ? 2 : 1; }
        out.mcol_cnt.push_back(mcnt ? (int)round_up(mcnt, 64) : 0);
        out.mcol_used.push_back(mcnt);
        kmq += out.mcol_cnt.back();
        (void)id;
    }
    out.n_class = (int)keep.size();
    out.Kq = kq;
    out.Kmq = kmq;
    std::vector<int> new_id(ncls, -1);
    for (int i = 0; i < out.n_class; ++i) new_id[keep[i]] = i;
    // pair columns
    out.pc_mu0.assign(kq, 0); out.pc_nu0.assign(kq, 0); out.pc_mu1.assign(kq, 0); out.pc_nu1.assign(kq, 0);
    out.pc_c0.assign(kq, 0.0); out.pc_c1.assign(kq, 0.0);
    out.pc_partner.assign(kq, -1);
    out.pc_re.assign(kq, 0.0); out.pc_im.assign(kq, 0.0); out.pc_zc.assign(kq, 0.0);
    long long total_cols = 0;
    for (const Comp &k : comps) {
        const int g = new_id[k.cls];
        const bool real = out.cls_real[g] != 0;
        const double sK = real ? (double)sub : 0.5 * sub;
        const int ncol = k.im.empty() ? 1 : 2;
        total_cols += ncol;
        for (int part = 0; part < ncol; ++part) {
            const int c = k.col + part;
            const std::vector<Term> &tm = part ? k.im : k.re;
            const double sg = (part && k.conj) ? -1.0 : 1.0;   // canonical = conjugate: imaginary part negated
            if (tm.size() > 0) { out.pc_mu0[c] = tm[0].mu; out.pc_nu0[c] = tm[0].nu; out.pc_c0[c] = sg * tm[0].c; }
            if (tm.size() > 1) { out.pc_mu1[c] = tm[1].mu; out.pc_nu1[c] = tm[1].nu; out.pc_c1[c] = sg * tm[1].c; }
            const double s = part ? -1.0 : 1.0;
            out.pc_partner[c] = ncol == 2 ? k.col + 1 - part : -1;
            out.pc_re[c] = sK * k.m;
            out.pc_im[c] = (real || ncol == 1) ? 0.0 : sK * k.m * s;
            out.pc_zc[c] = (real || ncol == 1) ? 0.0 : -s;
        }
    }
    if (total_cols != P) return 0;   // not a decomposition of the pair space (cannot happen for a valid analysis)
    // reconstruction of every packed pair
    auto packed = [n](int a, int b) {
        const long long lo = std::min(a, b), hi = std::max(a, b);
        return lo * n - lo * (lo - 1) / 2 + (hi - lo);
    };
    out.pp_col0.assign(P, 0); out.pp_col1.assign(P, 0);
    out.pp_c0.assign(P, 0.0); out.pp_c1.assign(P, 0.0);
    std::vector<int> nterm(P, 0);
    for (const Recon &r : recon) {
        const Comp &k = comps[r.comp];
        const long long p = packed(r.mu, r.nu);
        const int col = k.col + r.part;
        const double c = r.c * ((r.part && k.conj) ? -1.0 : 1.0);
        if (nterm[p] == 0) { out.pp_col0[p] = col; out.pp_c0[p] = c; }
        else if (nterm[p] == 1) { out.pp_col1[p] = col; out.pp_c1[p] = c; }
        else return 0;
        ++nterm[p];
    }
    for (long long p = 0; p < P; ++p)
        if (nterm[p] == 0) return 0;
    // mode columns
    out.mc_mode.assign(kmq, 0); out.mc_partner.assign(kmq, -1);
    out.mc_sign.assign(kmq, 0.0); out.mc_re.assign(kmq, 0.0); out.mc_im.assign(kmq, 0.0); out.mc_zc.assign(kmq, 0.0);
    out.mode_col.assign(n, -1);
    for (const ModeComp &mc : mcomps) {
        const int g = new_id[mc.cls];
        if (g < 0) continue;   // a class without pair components: its averages' terms vanish
        const bool real = out.cls_real[g] != 0;
        const double sK = real ? (double)sub : 0.5 * sub;
        const int ncol = mc.qb >= 0 ? 2 : 1;
        for (int part = 0; part < ncol; ++part) {
            const int c = mc.col + part;
            const double s = part ? -1.0 : 1.0;
            out.mc_mode[c] = part ? mc.qb : mc.q;
            out.mc_sign[c] = (part && mc.conj) ? -1.0 : 1.0;
            out.mc_partner[c] = ncol == 2 ? mc.col + 1 - part : -1;
            out.mc_re[c] = sK;
            out.mc_im[c] = (real || ncol == 1) ? 0.0 : sK * s;
            out.mc_zc[c] = (real || ncol == 1) ? 0.0 : -s;
            out.mode_col[out.mc_mode[c]] = c;
        }
    }
    // work of the class contractions relative to one over every symmetry and all pairs
    double work = 0.0;
    for (int g = 0; g < out.n_class; ++g) work += (out.cls_real[g] ? 1.0 : 2.0) * out.pcol_cnt[g];
    out.flops_ratio = work / ((double)sub * (double)P);
    out.ok = true;
    return 0;
}

}  // namespace tdscha

// ================================================================================================
// Device: tables, operands, left operands, reconstruction
// ================================================================================================
namespace tdscha {
namespace {

template <typename T>
int upload(const std::vector<T> &v, T **dst, size_t *acc) {
    *dst = nullptr;
    if (v.empty()) return 0;
    TD_CUDA(cudaMalloc(dst, v.size() * sizeof(T)));
    TD_CUDA(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    *acc += v.size() * sizeof(T);
    return 0;
}

__device__ __forceinline__ long long packed_of(int a, int b, int n) {
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    return (long long)lo * n - ((long long)lo * (lo - 1)) / 2 + (hi - lo);
}

unsigned grid1(long long work) { return (unsigned)std::max<long long>(1, std::min<long long>((work + 255) / 256, 148LL * 32)); }

// columns one per thread, rows in groups of rb (grid.y capped; the kernels stride over row groups)
dim3 grid_cols_rows(long long cols, long long rows, int rb) {
    const long long gx = std::max<long long>(1, ceil_div(cols, 256));
    const long long gy = std::max<long long>(1, std::min<long long>(ceil_div(rows, rb), 65535));
    return dim3((unsigned)gx, (unsigned)gy);
}

dim3 grid_rows(long long cols, long long rows) {
    const long long gx = std::max<long long>(1, std::min<long long>(ceil_div(cols, 256), 64));
    const long long gy = std::max<long long>(1, std::min<long long>(rows, 65535));
    return dim3((unsigned)gx, (unsigned)gy);
}

// Vq (2Nc x Kq) and VqT (Kq x N2pc) together: one CTA per 64 x 64 tile of (configuration rows,
// component columns) computes the tile once into shared memory (hi, lo) and writes it row-major and
// transposed, 128 bytes or more per warp on both sides.  Rows k >= 2Nc (up to N2pc) are zero in VqT.
template <typename T>
__device__ __forceinline__ void split_to(Format fmt, double v, T &h, T &l);
template <>
__device__ __forceinline__ void split_to<uint16_t>(Format, double v, uint16_t &h, uint16_t &l) {
    h = bf16_bits_rn((float)v);
    l = bf16_bits_rn((float)(v - (double)bf16_bits_to_float(h)));
}
template <>
__device__ __forceinline__ void split_to<float>(Format, double v, float &h, float &l) {
    h = tf32_round((float)v);
    l = tf32_round((float)(v - (double)h));
}
template <>
__device__ __forceinline__ void split_to<double>(Format, double v, double &h, double &l) {
    h = v;
    l = 0.0;
}

template <typename T>
__global__ void __launch_bounds__(256) build_Vq_tiles_kernel(const double *__restrict__ X, const double *__restrict__ G, int n,
                                                             long long Nc, long long N2pc, int Kq, const int *__restrict__ mu0,
                                                             const int *__restrict__ nu0, const int *__restrict__ mu1,
                                                             const int *__restrict__ nu1, const double *__restrict__ c0,
                                                             const double *__restrict__ c1, Format fmt, T *__restrict__ V_hi,
                                                             T *__restrict__ V_lo, T *__restrict__ VT_hi, T *__restrict__ VT_lo) {
    constexpr int LO_ROWS = sizeof(T) == 8 ? 1 : 64;   // FP64 has no lo part
    __shared__ T th[64][65];
    __shared__ T tl[LO_ROWS][65];
    const long long k0 = (long long)blockIdx.y * 64;   // configuration rows (of [x x^T ; sym(x g^T)])
    const int cb = blockIdx.x * 64;                     // component columns
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const bool lo = V_lo != nullptr;
    for (int e = tid; e < 64 * 64; e += 256) {
        const int r = e >> 6, cc = e & 63;
        const long long k = k0 + r;
        const int c = cb + cc;
        double v = 0.0;
        if (k < 2 * Nc && c < Kq) {
            const bool second = k >= Nc;
            const double *x = X + (second ? k - Nc : k) * n;
            const int a0 = mu0[c], b0 = nu0[c], a1 = mu1[c], b1 = nu1[c];
            if (!second) {
                v = c0[c] * x[a0] * x[b0] + c1[c] * x[a1] * x[b1];
            } else {
                const double *g = G + (k - Nc) * n;
                v = 0.5 * (c0[c] * (x[a0] * g[b0] + x[b0] * g[a0]) + c1[c] * (x[a1] * g[b1] + x[b1] * g[a1]));
            }
        }
        T h, l;
        split_to<T>(fmt, v, h, l);
        th[r][cc] = h;
        if constexpr (LO_ROWS == 64) tl[r][cc] = l;
    }
    __syncthreads();
    // row-major: rows k < 2Nc, 64 columns
    constexpr int EPW = sizeof(T) == 2 ? 2 : 1;   // elements per store word
    constexpr int WPR = 64 / EPW;                  // words per tile row
    for (int w = tid; w < 64 * WPR; w += 256) {
        const int r = w / WPR, j = (w % WPR) * EPW;
        const long long k = k0 + r;
        if (k >= 2 * Nc || cb + j >= Kq) continue;
        if constexpr (EPW == 2) {
            const uint32_t ph = (uint32_t)th[r][j] | ((uint32_t)th[r][j + 1] << 16);
            *reinterpret_cast<uint32_t *>(V_hi + k * Kq + cb + j) = ph;
            if (lo) *reinterpret_cast<uint32_t *>(V_lo + k * Kq + cb + j) = (uint32_t)tl[r][j] | ((uint32_t)tl[r][j + 1] << 16);
        } else {
            V_hi[k * Kq + cb + j] = th[r][j];
            if constexpr (LO_ROWS == 64)
                if (lo) V_lo[k * Kq + cb + j] = tl[r][j];
        }
    }
    // transposed: rows c (64), columns k0 .. k0 + 63 (< N2pc)
    if (VT_hi == nullptr) return;
    for (int w = tid; w < 64 * WPR; w += 256) {
        const int cr = w / WPR, j = (w % WPR) * EPW;
        const int c = cb + cr;
        const long long k = k0 + j;
        if (c >= Kq || k >= N2pc) continue;
        if constexpr (EPW == 2) {
            *reinterpret_cast<uint32_t *>(VT_hi + (long long)c * N2pc + k) = (uint32_t)th[j][cr] | ((uint32_t)th[j + 1][cr] << 16);
            if (lo)
                *reinterpret_cast<uint32_t *>(VT_lo + (long long)c * N2pc + k) =
                    (uint32_t)tl[j][cr] | ((uint32_t)tl[j + 1][cr] << 16);
        } else {
            VT_hi[(long long)c * N2pc + k] = th[j][cr];
            if constexpr (LO_ROWS == 64)
                if (lo) VT_lo[(long long)c * N2pc + k] = tl[j][cr];
        }
    }
}

// The same from the transposed ensemble XGT = [X^T ; G^T] (2n x ldT, configuration-contiguous): one
// CTA per (COLS component columns, 256 configuration rows of [x x^T ; sym(x g^T)]), one thread per
// configuration row; every read of XGT is a coalesced row segment, and consecutive CTAs share the
// same 256 configurations (x fastest), whose XGT block (2n x 256) stays in L2 while every column
// tile is built from it.  VqT rows go out directly (512 B per warp), Vq rows through shared memory.
template <typename T>
__global__ void __launch_bounds__(256, 2) build_Vq_cols_kernel(const double *__restrict__ XGT, long long ldT, int n, long long Nc,
                                                            long long N2pc, int Kq, const int *__restrict__ mu0,
                                                            const int *__restrict__ nu0, const int *__restrict__ mu1,
                                                            const int *__restrict__ nu1, const double *__restrict__ c0,
                                                            const double *__restrict__ c1, Format fmt, T *__restrict__ V_hi,
                                                            T *__restrict__ V_lo, T *__restrict__ VT_hi, T *__restrict__ VT_lo) {
    constexpr int COLS = sizeof(T) == 2 ? 64 : 32;   // 128 bytes of a Vq row
    constexpr int LDS = 257;                          // shared row length (conflict-free column reads)
    extern __shared__ __align__(16) uint8_t smem_raw[];
    T *th = reinterpret_cast<T *>(smem_raw);          // [COLS][LDS]
    T *tl = th + COLS * LDS;
    const int cb = blockIdx.x * COLS;
    const long long k0 = (long long)blockIdx.y * 256;
    const int t = threadIdx.x;
    const long long k = k0 + t;
    const bool lo = V_lo != nullptr;
    const bool second = k >= Nc && k < 2 * Nc;
    const bool live = k < 2 * Nc;
    const long long i = second ? k - Nc : k;
    // four columns per pass: every load of the pass is issued before the first is used, so the
    // XGT reads of the four columns overlap instead of waiting one after the other
    constexpr int U = 4;
    const double *Xr = XGT + i;                              // column i of every mode row
    const double *Gr = XGT + (long long)n * ldT + i;
    for (int cc0 = 0; cc0 < COLS; cc0 += U) {
        double v[U];
        if (live) {
            int a0[U], b0[U], a1[U], b1[U];
            double f0[U], f1[U], xa0[U], xb0[U], xa1[U], xb1[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = cb + cc0 + u;
                a0[u] = __ldg(mu0 + c); b0[u] = __ldg(nu0 + c); a1[u] = __ldg(mu1 + c); b1[u] = __ldg(nu1 + c);
                f0[u] = __ldg(c0 + c); f1[u] = __ldg(c1 + c);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                xa0[u] = Xr[(long long)a0[u] * ldT]; xb0[u] = Xr[(long long)b0[u] * ldT];
                xa1[u] = Xr[(long long)a1[u] * ldT]; xb1[u] = Xr[(long long)b1[u] * ldT];
            }
            if (!second) {
#pragma unroll
                for (int u = 0; u < U; ++u) v[u] = f0[u] * xa0[u] * xb0[u] + f1[u] * xa1[u] * xb1[u];
            } else {
                double ga0[U], gb0[U], ga1[U], gb1[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    ga0[u] = Gr[(long long)a0[u] * ldT]; gb0[u] = Gr[(long long)b0[u] * ldT];
                    ga1[u] = Gr[(long long)a1[u] * ldT]; gb1[u] = Gr[(long long)b1[u] * ldT];
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
                    v[u] = 0.5 * (f0[u] * (xa0[u] * gb0[u] + xb0[u] * ga0[u]) + f1[u] * (xa1[u] * gb1[u] + xb1[u] * ga1[u]));
            }
        } else {
#pragma unroll
            for (int u = 0; u < U; ++u) v[u] = 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int cc = cc0 + u, c = cb + cc;
            T h, l;
            split_to<T>(fmt, v[u], h, l);
            if (VT_hi && k < N2pc) {
                VT_hi[(long long)c * N2pc + k] = h;
                if (lo) VT_lo[(long long)c * N2pc + k] = l;
            }
            th[cc * LDS + t] = h;
            tl[cc * LDS + t] = l;
        }
    }
    __syncthreads();
    // Vq rows k < 2Nc: one warp per row and pass, COLS columns as 32-bit words
    constexpr int EPW = sizeof(T) == 2 ? 2 : 1;
    constexpr int WPR = COLS / EPW;   // = 32
    const int warp = t >> 5, lane = t & 31;
    for (int r = warp; r < 256; r += 8) {
        const long long kr = k0 + r;
        if (kr >= 2 * Nc) break;
        const int j = lane * EPW;
        if constexpr (EPW == 2) {
            *reinterpret_cast<uint32_t *>(V_hi + kr * Kq + cb + j) =
                (uint32_t)th[j * LDS + r] | ((uint32_t)th[(j + 1) * LDS + r] << 16);
            if (lo)
                *reinterpret_cast<uint32_t *>(V_lo + kr * Kq + cb + j) =
                    (uint32_t)tl[j * LDS + r] | ((uint32_t)tl[(j + 1) * LDS + r] << 16);
        } else {
            V_hi[kr * Kq + cb + j] = th[j * LDS + r];
            if (lo) V_lo[kr * Kq + cb + j] = tl[j * LDS + r];
        }
        static_assert(WPR == 32, "one warp per Vq row");
    }
}

template <typename T>
int build_Vq_cols(const FreqTables &t, const double *XGT, long long ldT, int n, long long Nc, long long N2pc, Format fmt,
                  void *V_hi, void *V_lo, void *VT_hi, void *VT_lo, cudaStream_t st) {
    constexpr int COLS = sizeof(T) == 2 ? 64 : 32;
    TD_CHECK(t.Kq % COLS == 0 && N2pc % 64 == 0 && ceil_div(N2pc, 256) <= 65535, TDSCHA_EINVAL, "operand build: %lld x %d",
             N2pc, t.Kq);
    const size_t smem = (size_t)2 * COLS * 257 * sizeof(T);
    auto kern = build_Vq_cols_kernel<T>;
    TD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const dim3 grid((unsigned)(t.Kq / COLS), (unsigned)ceil_div(N2pc, 256));
    kern<<<grid, 256, smem, st>>>(XGT, ldT, n, Nc, N2pc, t.Kq, t.pc_mu0, t.pc_nu0, t.pc_mu1, t.pc_nu1, t.pc_c0, t.pc_c1, fmt,
                                  static_cast<T *>(V_hi), static_cast<T *>(V_lo), static_cast<T *>(VT_hi), static_cast<T *>(VT_lo));
    TD_CUDA(cudaGetLastError());
    return 0;
}

template <typename T>
int build_Vq_tiles(const FreqTables &t, const double *X, const double *G, int n, long long Nc, long long N2pc, Format fmt,
                   void *V_hi, void *V_lo, void *VT_hi, void *VT_lo, cudaStream_t st) {
    TD_CHECK(N2pc % 64 == 0 && N2pc / 64 <= 65535 && t.Kq % 64 == 0, TDSCHA_EINVAL, "operand tiles: %lld x %d", N2pc, t.Kq);
    const dim3 grid((unsigned)(t.Kq / 64), (unsigned)(N2pc / 64));
    build_Vq_tiles_kernel<T><<<grid, dim3(32, 8), 0, st>>>(X, G, n, Nc, N2pc, t.Kq, t.pc_mu0, t.pc_nu0, t.pc_mu1, t.pc_nu1, t.pc_c0,
                                                           t.pc_c1, fmt, static_cast<T *>(V_hi), static_cast<T *>(V_lo),
                                                           static_cast<T *>(VT_hi), static_cast<T *>(VT_lo));
    TD_CUDA(cudaGetLastError());
    return 0;
}

// XGq (2Nc x Kmq): mode components of x (rows < Nc) and g
__global__ void build_XGq_kernel(const double *__restrict__ X, const double *__restrict__ G, int n, long long Nc, int Kmq,
                                 const int *__restrict__ mode, const double *__restrict__ sign, Format fmt, void *hi, void *lo) {
    const long long total = 2 * Nc * Kmq;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const long long k = idx / Kmq;
        const int c = (int)(idx - k * Kmq);
        const double v = k < Nc ? X[k * n + mode[c]] : G[(k - Nc) * n + mode[c]];
        store_split(fmt, hi, lo, idx, sign[c] * v);
    }
}

// YXq (Kmq x N2pc): mode components of y (columns < Nc) and of x~, zero past 2Nc
__global__ void build_YXq_kernel(const double *__restrict__ Y, const double *__restrict__ Xt, int n, long long Nc, long long N2pc,
                                 int Kmq, const int *__restrict__ mode, const double *__restrict__ sign, Format fmt, void *hi,
                                 void *lo) {
    const long long total = (long long)Kmq * N2pc;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const long long c = idx / N2pc, k = idx - c * N2pc;
        double v = 0.0;
        if (k < Nc) v = Y[k * n + mode[c]];
        else if (k < 2 * Nc) v = Xt[(k - Nc) * n + mode[c]];
        store_split(fmt, hi, lo, idx, sign[c] * v);
    }
}

// Lab rows r (real parts) and NR + r (imaginary parts) from the representatives' U rows.  One thread
// per component column c and LEFT_RB consecutive rows: the column's tables (packed indices, weights,
// partner) are read once and its LEFT_RB rows' gathers are independent, in flight together.
constexpr int LEFT_RB = 8;

template <typename InT>
__global__ void __launch_bounds__(256) left_ab_kernel(int NR, int n, int Kq, const InT *__restrict__ U, long long ldu,
                                                      const int *__restrict__ mu0, const int *__restrict__ nu0,
                                                      const int *__restrict__ mu1, const int *__restrict__ nu1,
                                                      const double *__restrict__ c0, const double *__restrict__ c1,
                                                      const int *__restrict__ partner, const double *__restrict__ re,
                                                      const double *__restrict__ im, Format fmt, void *hi, void *lo) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Kq) return;
    const long long p0 = packed_of(mu0[c], nu0[c], n), p1 = packed_of(mu1[c], nu1[c], n);
    const double a0 = c0[c], a1 = c1[c], rc = re[c], ic = im[c];
    const int pc = partner[c];
    const bool has = pc >= 0 && ic != 0.0;
    long long q0 = 0, q1 = 0;
    double b0 = 0.0, b1 = 0.0;
    if (has) {
        q0 = packed_of(mu0[pc], nu0[pc], n);
        q1 = packed_of(mu1[pc], nu1[pc], n);
        b0 = c0[pc];
        b1 = c1[pc];
    }
    for (long long r0 = (long long)blockIdx.y * LEFT_RB; r0 < NR; r0 += (long long)gridDim.y * LEFT_RB) {
#pragma unroll
        for (int i = 0; i < LEFT_RB; ++i) {
            const long long r = r0 + i;
            if (r >= NR) break;
            const InT *u = U + r * ldu;
            const double own = a0 * (double)u[p0] + a1 * (double)u[p1];
            const double oth = has ? b0 * (double)u[q0] + b1 * (double)u[q1] : 0.0;
            store_split(fmt, hi, lo, r * Kq + c, rc * own);
            store_split(fmt, hi, lo, (NR + r) * Kq + c, ic * oth);
        }
    }
}

template <typename InT>
__global__ void left_cd_kernel(int NR, int Kmq, const InT *__restrict__ r1p, long long ldr, const int *__restrict__ mode,
                               const double *__restrict__ sign, const int *__restrict__ partner, const double *__restrict__ re,
                               const double *__restrict__ im, Format fmt, void *hi, void *lo) {
    const long long total = (long long)NR * Kmq;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const long long r = idx / Kmq;
        const int c = (int)(idx - r * Kmq);
        const InT *v = r1p + r * ldr;
        const double own = sign[c] * (double)v[mode[c]];
        const int pc = partner[c];
        const double oth = (pc >= 0 && im[c] != 0.0) ? sign[pc] * (double)v[mode[pc]] : 0.0;
        store_split(fmt, hi, lo, r * Kmq + c, re[c] * own);
        store_split(fmt, hi, lo, (NR + r) * Kmq + c, im[c] * oth);
    }
}

template <typename AccT>
__device__ __forceinline__ double own_out(const AccT *o1, const AccT *o2, int c, const int *partner, const double *zc) {
    double v = (double)o1[c];
    const double z = zc[c];
    if (z != 0.0) v += z * (double)o2[partner[c]];
    return v;
}

// Zs rows from the class outputs: one thread per pair p and LEFT_RB consecutive rows, the pair's
// tables (columns, weights, partners) read once
template <typename AccT>
__global__ void __launch_bounds__(256) recon_z_kernel(int NR, long long P, int Kq, const AccT *__restrict__ O,
                                                      const int *__restrict__ pmu, const int *__restrict__ pnu,
                                                      const int *__restrict__ col0, const int *__restrict__ col1,
                                                      const double *__restrict__ pc0, const double *__restrict__ pc1,
                                                      const int *__restrict__ partner, const double *__restrict__ zc,
                                                      AccT *__restrict__ Zs, long long ldz) {
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= P) return;
    const int ca = col0[p], cb = col1[p];
    const double k0 = pc0[p], k1 = pc1[p], fac = pmu[p] == pnu[p] ? 1.0 : 2.0;
    const double za = zc[ca], zb = k1 != 0.0 ? zc[cb] : 0.0;
    const int qa = za != 0.0 ? partner[ca] : 0, qb = zb != 0.0 ? partner[cb] : 0;
    for (long long r0 = (long long)blockIdx.y * LEFT_RB; r0 < NR; r0 += (long long)gridDim.y * LEFT_RB) {
#pragma unroll
        for (int i = 0; i < LEFT_RB; ++i) {
            const long long r = r0 + i;
            if (r >= NR) break;
            const AccT *o1 = O + r * Kq, *o2 = O + (NR + r) * Kq;
            double va = (double)o1[ca];
            if (za != 0.0) va += za * (double)o2[qa];
            double v = k0 * va;
            if (k1 != 0.0) {
                double vb = (double)o1[cb];
                if (zb != 0.0) vb += zb * (double)o2[qb];
                v += k1 * vb;
            }
            Zs[r * ldz + p] = (AccT)(fac * v);
        }
    }
}

template <typename AccT>
__global__ void recon_f_kernel(int NR, int n, int Kmq, const AccT *__restrict__ OF, const int *__restrict__ mode_col,
                               const double *__restrict__ sign, const int *__restrict__ partner, const double *__restrict__ zc,
                               AccT *__restrict__ Fs, long long ldf) {
    const long long total = (long long)NR * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const long long r = idx / n;
        const int m = (int)(idx - r * n);
        const int c = mode_col[m];
        double v = 0.0;
        if (c >= 0) v = sign[c] * own_out(OF + r * Kmq, OF + (NR + r) * Kmq, c, partner, zc);
        Fs[r * ldf + m] = (AccT)v;
    }
}

// 4 consecutive values into an operand slot of format fmt (fp32 arithmetic; idx a multiple of 4)
__device__ __forceinline__ void store4_split(Format fmt, void *hi, void *lo, long long idx, const float (&v)[4]) {
    if (fmt == FMT_BF16) {
        __nv_bfloat16 h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            h[e] = __float2bfloat16_rn(v[e]);
            l[e] = __float2bfloat16_rn(v[e] - __bfloat162float(h[e]));
        }
        *reinterpret_cast<uint2 *>(static_cast<__nv_bfloat16 *>(hi) + idx) = *reinterpret_cast<const uint2 *>(h);
        if (lo) *reinterpret_cast<uint2 *>(static_cast<__nv_bfloat16 *>(lo) + idx) = *reinterpret_cast<const uint2 *>(l);
    } else {
        float4 h, l;
        h.x = tf32_round(v[0]); h.y = tf32_round(v[1]); h.z = tf32_round(v[2]); h.w = tf32_round(v[3]);
        l.x = tf32_round(v[0] - h.x); l.y = tf32_round(v[1] - h.y); l.z = tf32_round(v[2] - h.z); l.w = tf32_round(v[3] - h.w);
        *reinterpret_cast<float4 *>(static_cast<float *>(hi) + idx) = h;
        if (lo) *reinterpret_cast<float4 *>(static_cast<float *>(lo) + idx) = l;
    }
}

// One CTA row per operand row (grid-stride), threads over quads of configurations.  vec: fp32
// accumulators, a split format and Nc a multiple of 4 (aligned vector loads and stores).
template <typename AccT, bool VEC>
__global__ void __launch_bounds__(256) freq_weights_kernel(const AccT *__restrict__ H, const AccT *__restrict__ Ch, long long ld,
                                                           const double *__restrict__ rho, long long Nc, int NR, long long rows,
                                                           const int *__restrict__ cls_real, long long N2pc, int d4, Format fmt,
                                                           void *Cw_hi, void *Cw_lo, void *AB_hi, void *AB_lo) {
    for (long long r = blockIdx.y; r < rows; r += gridDim.y) {
        const long long g = r / (2LL * NR);
        if (r - g * 2LL * NR >= NR && cls_real[g]) continue;   // imaginary row of a real class
        const AccT *h = H + r * ld, *c = Ch + r * ld;
        const long long o = r * N2pc;
        if constexpr (VEC) {
            const float k4 = d4 ? 1.f : 0.f;
            for (long long i0 = 4LL * (blockIdx.x * (long long)blockDim.x + threadIdx.x); i0 < Nc;
                 i0 += 4LL * gridDim.x * blockDim.x) {
                const float4 a = *reinterpret_cast<const float4 *>(h + i0), b = *reinterpret_cast<const float4 *>(h + Nc + i0);
                const float4 cc = *reinterpret_cast<const float4 *>(c + i0), dd = *reinterpret_cast<const float4 *>(c + Nc + i0);
                const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
                const float cv[4] = {cc.x, cc.y, cc.z, cc.w}, dv[4] = {dd.x, dd.y, dd.z, dd.w};
                float half_delta[4], gamma[4], alpha[4], beta[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float rh = (float)rho[i0 + e];
                    gamma[e] = rh * (-cv[e] * (1.f / 3.f) + k4 * av[e] * 0.125f);
                    half_delta[e] = 0.5f * rh * (-dv[e] * (1.f / 3.f) + k4 * bv[e] * 0.25f);
                    alpha[e] = -rh * av[e] * (1.f / 6.f);
                    beta[e] = -rh * bv[e] * (1.f / 3.f);
                }
                store4_split(fmt, Cw_hi, Cw_lo, o + i0, half_delta);
                store4_split(fmt, Cw_hi, Cw_lo, o + Nc + i0, gamma);
                store4_split(fmt, AB_hi, AB_lo, o + i0, alpha);
                store4_split(fmt, AB_hi, AB_lo, o + Nc + i0, beta);
            }
        } else {
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < Nc; i += (long long)gridDim.x * blockDim.x) {
                const double a = (double)h[i], b = (double)h[Nc + i], cv = (double)c[i], dv = (double)c[Nc + i];
                const double rh = rho[i];
                const double gam = rh * (-cv / 3.0 + (d4 ? a / 8.0 : 0.0));
                const double del = rh * (-dv / 3.0 + (d4 ? b / 4.0 : 0.0));
                store_split(fmt, Cw_hi, Cw_lo, o + i, 0.5 * del);
                store_split(fmt, Cw_hi, Cw_lo, o + Nc + i, gam);
                store_split(fmt, AB_hi, AB_lo, o + i, -rh * a / 6.0);
                store_split(fmt, AB_hi, AB_lo, o + Nc + i, -rh * b / 3.0);
            }
        }
        // zero columns past 2Nc (the contractions' K runs to N2pc)
        if (blockIdx.x == 0)
            for (long long k = 2 * Nc + threadIdx.x; k < N2pc; k += blockDim.x) {
                store_split(fmt, Cw_hi, Cw_lo, o + k, 0.0);
                store_split(fmt, AB_hi, AB_lo, o + k, 0.0);
            }
    }
}

template <Format FMT>
__device__ __forceinline__ float split_value(const void *hi, const void *lo, long long idx) {
    if constexpr (FMT == FMT_BF16) {
        float v = bf16_bits_to_float(static_cast<const uint16_t *>(hi)[idx]);
        if (lo) v += bf16_bits_to_float(static_cast<const uint16_t *>(lo)[idx]);
        return v;
    } else {
        float v = static_cast<const float *>(hi)[idx];
        if (lo) v += static_cast<const float *>(lo)[idx];
        return v;
    }
}

// One CTA per (32 rows of one class, 128 configurations): the class's mode components of the
// configurations (x and g) and of the rows' left operands in shared memory (fp32, padded to 65
// columns), then per (row, configuration) the dot products c, d and the weights.
template <Format FMT>
__global__ void __launch_bounds__(256) weights_cd_kernel(const float *__restrict__ H, long long ld, const void *Lcd_hi,
                                                         const void *Lcd_lo, const void *XG_hi, const void *XG_lo, int Kmq,
                                                         const double *__restrict__ rho, long long Nc, int NR, int tiles_per_class,
                                                         const int *__restrict__ cls_real, const int *__restrict__ mcol_off,
                                                         const int *__restrict__ mcol_used, long long N2pc, int d4, void *Cw_hi,
                                                         void *Cw_lo, void *AB_hi, void *AB_lo) {
    extern __shared__ __align__(16) float wsm[];
    float *Xs = wsm;                   // [128][65]
    float *Gs = Xs + 128 * 65;         // [128][65]
    float *Ls = Gs + 128 * 65;         // [32][65]
    const int g = blockIdx.y;
    const int Kc = mcol_used[g], moff = mcol_off[g];
    const bool real_cls = cls_real[g] != 0;
    const int rows_cls = real_cls ? NR : 2 * NR;
    const long long i0 = (long long)blockIdx.x * 128;
    const int tid = threadIdx.x;
    for (int e = tid; e < 128 * 64; e += 256) {
        const int ii = e >> 6, cc = e & 63;
        const long long i = i0 + ii;
        float xv = 0.f, gv = 0.f;
        if (cc < Kc && i < Nc) {
            xv = split_value<FMT>(XG_hi, XG_lo, i * Kmq + moff + cc);
            gv = split_value<FMT>(XG_hi, XG_lo, (Nc + i) * Kmq + moff + cc);
        }
        Xs[ii * 65 + cc] = xv;
        Gs[ii * 65 + cc] = gv;
    }
    const int warp = tid >> 5, lane = tid & 31;
    const float k4 = d4 ? 1.f : 0.f;
    // the configuration slice stays in shared memory while the CTA walks every row tile of the class
    for (int tb = 0; tb * 32 < rows_cls; ++tb) {
    __syncthreads();
    for (int e = tid; e < 32 * 64; e += 256) {
        const int rr = e >> 6, cc = e & 63;
        const int lr = tb * 32 + rr;   // row inside the class: comp * NR + j
        float v = 0.f;
        if (cc < Kc && lr < rows_cls) v = split_value<FMT>(Lcd_hi, Lcd_lo, (long long)lr * Kmq + moff + cc);
        Ls[rr * 65 + cc] = v;
    }
    __syncthreads();
    for (int rr = warp; rr < 32; rr += 8) {
        const int lr = tb * 32 + rr;
        if (lr >= rows_cls) break;
        const long long r = (long long)g * 2 * NR + lr;
        const float *h = H + r * ld;
        const float *l = Ls + rr * 65;
        for (int q = 0; q < 4; ++q) {
            const int ii = lane + 32 * q;
            const long long i = i0 + ii;
            if (i >= Nc) break;
            const float *xs = Xs + ii * 65, *gs = Gs + ii * 65;
            float c = 0.f, d = 0.f;
            for (int cc = 0; cc < Kc; ++cc) {
                c = fmaf(l[cc], xs[cc], c);
                d = fmaf(l[cc], gs[cc], d);
            }
            const float a = h[i], b = h[Nc + i];
            const float rh = (float)rho[i];
            const float gam = rh * (-c * (1.f / 3.f) + k4 * a * 0.125f);
            const float hdel = 0.5f * rh * (-d * (1.f / 3.f) + k4 * b * 0.25f);
            const long long o = r * N2pc;
            store_split(FMT, Cw_hi, Cw_lo, o + i, (double)hdel);
            store_split(FMT, Cw_hi, Cw_lo, o + Nc + i, (double)gam);
            store_split(FMT, AB_hi, AB_lo, o + i, (double)(-rh * a * (1.f / 6.f)));
            store_split(FMT, AB_hi, AB_lo, o + Nc + i, (double)(-rh * b * (1.f / 3.f)));
        }
        if (blockIdx.x == 0)
            for (long long k = 2 * Nc + lane; k < N2pc; k += 32) {
                store_split(FMT, Cw_hi, Cw_lo, r * N2pc + k, 0.0);
                store_split(FMT, AB_hi, AB_lo, r * N2pc + k, 0.0);
            }
    }
    }
}

}  // namespace

template <typename AccT>
int freq_weights(const FreqTables &t, const AccT *H, const AccT *Ch, long long ld, const double *rho, long long Nc, int NR,
                 long long N2pc, int d4, Format fmt, void *Cw_hi, void *Cw_lo, void *AB_hi, void *AB_lo, cudaStream_t st) {
    const long long rows = (long long)t.n_class * 2 * NR;
    const bool vec = sizeof(AccT) == 4 && fmt != FMT_F64 && Nc % 4 == 0 && ld % 4 == 0;
    const long long per = vec ? ceil_div(Nc, 4) : Nc;
    const dim3 grid((unsigned)std::max<long long>(1, std::min<long long>(ceil_div(per, 256), 64)),
                    (unsigned)std::max<long long>(1, std::min<long long>(rows, 65535)));
    if (vec)
        freq_weights_kernel<AccT, true><<<grid, 256, 0, st>>>(H, Ch, ld, rho, Nc, NR, rows, t.d_cls_real, N2pc, d4, fmt, Cw_hi,
                                                              Cw_lo, AB_hi, AB_lo);
    else
        freq_weights_kernel<AccT, false><<<grid, 256, 0, st>>>(H, Ch, ld, rho, Nc, NR, rows, t.d_cls_real, N2pc, d4, fmt, Cw_hi,
                                                               Cw_lo, AB_hi, AB_lo);
    TD_CUDA(cudaGetLastError());
    return 0;
}

int freq_weights_cd(const FreqTables &t, const float *H, long long ld, const void *Lcd_hi, const void *Lcd_lo, const void *XG_hi,
                    const void *XG_lo, const double *rho, long long Nc, int NR, long long N2pc, int d4, Format fmt, void *Cw_hi,
                    void *Cw_lo, void *AB_hi, void *AB_lo, cudaStream_t st) {
    TD_CHECK(fmt == FMT_BF16 || fmt == FMT_TF32, TDSCHA_EINVAL, "fused weights need a split format");
    TD_CHECK(t.Kmq > 0, TDSCHA_EINVAL, "fused weights need mode columns");
    const int tiles_per_class = ceil_div(2 * NR, 32);
    const long long gy = t.n_class;
    const size_t smem = (size_t)(2 * 128 + 32) * 65 * sizeof(float);
    const dim3 grid((unsigned)ceil_div(Nc, 128), (unsigned)gy);
    if (fmt == FMT_BF16) {
        TD_CUDA(cudaFuncSetAttribute(weights_cd_kernel<FMT_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        weights_cd_kernel<FMT_BF16><<<grid, 256, smem, st>>>(H, ld, Lcd_hi, Lcd_lo, XG_hi, XG_lo, t.Kmq, rho, Nc, NR, tiles_per_class,
                                                             t.d_cls_real, t.d_mcol_off, t.d_mcol_used, N2pc, d4, Cw_hi, Cw_lo,
                                                             AB_hi, AB_lo);
    } else {
        TD_CUDA(cudaFuncSetAttribute(weights_cd_kernel<FMT_TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        weights_cd_kernel<FMT_TF32><<<grid, 256, smem, st>>>(H, ld, Lcd_hi, Lcd_lo, XG_hi, XG_lo, t.Kmq, rho, Nc, NR, tiles_per_class,
                                                             t.d_cls_real, t.d_mcol_off, t.d_mcol_used, N2pc, d4, Cw_hi, Cw_lo,
                                                             AB_hi, AB_lo);
    }
    TD_CUDA(cudaGetLastError());
    return 0;
}

template int freq_weights<float>(const FreqTables &, const float *, const float *, long long, const double *, long long, int,
                                 long long, int, Format, void *, void *, void *, void *, cudaStream_t);
template int freq_weights<double>(const FreqTables &, const double *, const double *, long long, const double *, long long,
                                  int, long long, int, Format, void *, void *, void *, void *, cudaStream_t);

int freq_tables_create(const FreqLayout &L, FreqTables **out) {
    *out = nullptr;
    auto *t = new FreqTables();
    t->n_class = L.n_class;
    t->Kq = L.Kq;
    t->Kmq = L.Kmq;
    t->cls_real = L.cls_real;
    t->pcol_off = L.pcol_off;
    t->pcol_cnt = L.pcol_cnt;
    t->mcol_off = L.mcol_off;
    t->mcol_cnt = L.mcol_cnt;
    t->mcol_used = L.mcol_used;
    t->flops_ratio = L.flops_ratio;
    size_t acc = 0;
    int rc = 0;
    if ((rc = upload(L.pc_mu0, &t->pc_mu0, &acc)) || (rc = upload(L.pc_nu0, &t->pc_nu0, &acc)) ||
        (rc = upload(L.pc_mu1, &t->pc_mu1, &acc)) || (rc = upload(L.pc_nu1, &t->pc_nu1, &acc)) ||
        (rc = upload(L.pc_partner, &t->pc_partner, &acc)) || (rc = upload(L.pc_c0, &t->pc_c0, &acc)) ||
        (rc = upload(L.pc_c1, &t->pc_c1, &acc)) || (rc = upload(L.pc_re, &t->pc_re, &acc)) ||
        (rc = upload(L.pc_im, &t->pc_im, &acc)) || (rc = upload(L.pc_zc, &t->pc_zc, &acc)) ||
        (rc = upload(L.pp_col0, &t->pp_col0, &acc)) || (rc = upload(L.pp_col1, &t->pp_col1, &acc)) ||
        (rc = upload(L.pp_c0, &t->pp_c0, &acc)) || (rc = upload(L.pp_c1, &t->pp_c1, &acc)) ||
        (rc = upload(L.mc_mode, &t->mc_mode, &acc)) || (rc = upload(L.mc_partner, &t->mc_partner, &acc)) ||
        (rc = upload(L.mode_col, &t->mode_col, &acc)) || (rc = upload(L.mc_sign, &t->mc_sign, &acc)) ||
        (rc = upload(L.mc_re, &t->mc_re, &acc)) || (rc = upload(L.mc_im, &t->mc_im, &acc)) ||
        (rc = upload(L.mc_zc, &t->mc_zc, &acc)) || (rc = upload(L.cls_real, &t->d_cls_real, &acc)) ||
        (rc = upload(L.mcol_off, &t->d_mcol_off, &acc)) || (rc = upload(L.mcol_used, &t->d_mcol_used, &acc))) {
        freq_tables_destroy(t);
        return rc;
    }
    t->bytes = acc;
    *out = t;
    return 0;
}

void freq_tables_destroy(FreqTables *t) {
    if (!t) return;
    void *ps[] = {t->pc_mu0, t->pc_nu0, t->pc_mu1, t->pc_nu1, t->pc_partner, t->pc_c0, t->pc_c1, t->pc_re, t->pc_im, t->pc_zc,
                  t->pp_col0, t->pp_col1, t->pp_c0, t->pp_c1, t->mc_mode, t->mc_partner, t->mode_col, t->mc_sign, t->mc_re,
                  t->mc_im, t->mc_zc, t->d_cls_real, t->d_mcol_off, t->d_mcol_used};
    for (void *p : ps)
        if (p) cudaFree(p);
    delete t;
}

size_t freq_operand_bytes(const FreqTables &t, long long Nc, Format fmt, bool lo) {
    const long long N2pc = round_up(2 * Nc, 64);
    const size_t per = (size_t)(2 * Nc * t.Kq + (long long)t.Kq * N2pc + 2 * Nc * t.Kmq + (long long)t.Kmq * N2pc);
    return per * format_bytes(fmt) * (lo ? 2 : 1) + 8 * 256;
}

int freq_build_operands(const FreqTables &t, const double *X, const double *G, const double *Y, const double *Xt,
                        const double *XGT, long long ldT, int n, long long Nc, Format fmt, bool lo, void *buf, FreqOps &o,
                        cudaStream_t st) {
    const size_t es = format_bytes(fmt);
    const long long N2pc = round_up(2 * Nc, 64);
    const long long nV = 2 * Nc * t.Kq, nVT = (long long)t.Kq * N2pc, nXG = 2 * Nc * t.Kmq, nYX = (long long)t.Kmq * N2pc;
    uint8_t *b = static_cast<uint8_t *>(buf);
    size_t off = 0;
    auto take = [&](long long count) { void *p = b + off; off += ((size_t)count * es + 255) / 256 * 256; return p; };
    o = FreqOps();
    o.V_hi = take(nV);
    o.VT_hi = take(nVT);
    o.XG_hi = take(nXG);
    o.YX_hi = take(nYX);
    if (lo) {
        o.V_lo = take(nV);
        o.VT_lo = take(nVT);
        o.XG_lo = take(nXG);
        o.YX_lo = take(nYX);
    }
    // Vq and its transpose from shared-memory tiles (gathering the transpose from the ensemble per
    // component would re-read the ensemble rows once per component)
    // (from the transposed ensemble XGT when given: coalesced, L2-resident reads per configuration
    // block; else gathering from the ensemble rows)
    if (XGT && fmt == FMT_BF16)
        TD_TRY(build_Vq_cols<uint16_t>(t, XGT, ldT, n, Nc, N2pc, fmt, o.V_hi, o.V_lo, o.VT_hi, o.VT_lo, st));
    else if (XGT && fmt == FMT_TF32)
        TD_TRY(build_Vq_cols<float>(t, XGT, ldT, n, Nc, N2pc, fmt, o.V_hi, o.V_lo, o.VT_hi, o.VT_lo, st));
    else if (fmt == FMT_BF16)
        TD_TRY(build_Vq_tiles<uint16_t>(t, X, G, n, Nc, N2pc, fmt, o.V_hi, o.V_lo, o.VT_hi, o.VT_lo, st));
    else if (fmt == FMT_F64)
        TD_TRY(build_Vq_tiles<double>(t, X, G, n, Nc, N2pc, fmt, o.V_hi, nullptr, o.VT_hi, nullptr, st));
    else
        TD_TRY(build_Vq_tiles<float>(t, X, G, n, Nc, N2pc, fmt, o.V_hi, o.V_lo, o.VT_hi, o.VT_lo, st));
    build_XGq_kernel<<<grid1(nXG), 256, 0, st>>>(X, G, n, Nc, t.Kmq, t.mc_mode, t.mc_sign, fmt, o.XG_hi, o.XG_lo);
    build_YXq_kernel<<<grid1(nYX), 256, 0, st>>>(Y, Xt, n, Nc, N2pc, t.Kmq, t.mc_mode, t.mc_sign, fmt, o.YX_hi, o.YX_lo);
    TD_CUDA(cudaGetLastError());
    o.built = true;
    o.has_lo = lo;
    o.bytes = off;
    return 0;
}

template <typename InT>
int freq_left(const FreqTables &t, int NR, int n, const InT *U, long long ldu, const InT *r1p, long long ldr, Format fmt,
              void *Lab_hi, void *Lab_lo, void *Lcd_hi, void *Lcd_lo, cudaStream_t st) {
    left_ab_kernel<InT><<<grid_cols_rows(t.Kq, NR, LEFT_RB), 256, 0, st>>>(NR, n, t.Kq, U, ldu, t.pc_mu0, t.pc_nu0, t.pc_mu1, t.pc_nu1, t.pc_c0,
                                                             t.pc_c1, t.pc_partner, t.pc_re, t.pc_im, fmt, Lab_hi, Lab_lo);
    if (t.Kmq > 0)
        left_cd_kernel<InT><<<grid1((long long)NR * t.Kmq), 256, 0, st>>>(NR, t.Kmq, r1p, ldr, t.mc_mode, t.mc_sign, t.mc_partner,
                                                                         t.mc_re, t.mc_im, fmt, Lcd_hi, Lcd_lo);
    TD_CUDA(cudaGetLastError());
    return 0;
}

template <typename AccT>
int freq_reconstruct(const FreqTables &t, int NR, int n, long long P, const int *pmu, const int *pnu, const AccT *O,
                     const AccT *OF, AccT *Zs, long long ldz, AccT *Fs, long long ldf, cudaStream_t st) {
    recon_z_kernel<AccT><<<grid_cols_rows(P, NR, LEFT_RB), 256, 0, st>>>(NR, P, t.Kq, O, pmu, pnu, t.pp_col0, t.pp_col1, t.pp_c0, t.pp_c1,
                                                           t.pc_partner, t.pc_zc, Zs, ldz);
    recon_f_kernel<AccT><<<grid1((long long)NR * n), 256, 0, st>>>(NR, n, t.Kmq, OF, t.mode_col, t.mc_sign, t.mc_partner,
                                                                    t.mc_zc, Fs, ldf);
    TD_CUDA(cudaGetLastError());
    return 0;
}

template int freq_left<float>(const FreqTables &, int, int, const float *, long long, const float *, long long, Format, void *,
                              void *, void *, void *, cudaStream_t);
template int freq_left<double>(const FreqTables &, int, int, const double *, long long, const double *, long long, Format,
                               void *, void *, void *, void *, cudaStream_t);
template int freq_reconstruct<float>(const FreqTables &, int, int, long long, const int *, const int *, const float *,
                                     const float *, float *, long long, float *, long long, cudaStream_t);
template int freq_reconstruct<double>(const FreqTables &, int, int, long long, const int *, const int *, const double *,
                                      const double *, double *, long long, double *, long long, cudaStream_t);

}  // namespace tdscha

// ================================================================================================
// The averages' VJP in the character basis (device)
// ================================================================================================
namespace tdscha {
namespace {

template <typename T>
__global__ void transpose_left_kernel(const T *__restrict__ L, int NR, int NRp, long long cols, T *__restrict__ out) {
    __shared__ T tile[32][33];
    const long long c0 = (long long)blockIdx.x * 32;
    const int q0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int q = q0 + j, comp = q / NRp, jj = q - comp * NRp;
        const long long c = c0 + threadIdx.x;
        T v = T(0);
        if (comp < 2 && jj < NR && c < cols) v = L[(long long)(comp * NR + jj) * cols + c];
        tile[j][threadIdx.x] = v;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const long long c = c0 + j;
        const int q = q0 + threadIdx.x;
        if (c < cols && q < 2 * NRp) out[c * (2LL * NRp) + q] = tile[threadIdx.x][j];
    }
}

// One thread per (row r, configuration i) of a 32 x 32 tile; TRANS: the K's go out transposed
// through shared memory (coalesced along the rows).
template <typename AccT, bool TRANS>
__global__ void __launch_bounds__(256) vjp_coef_class_kernel(const AccT *__restrict__ H, const AccT *__restrict__ Ch,
                                                             const AccT *__restrict__ HQ, const AccT *__restrict__ Cp,
                                                             long long ld, int N, long long rows, int NR, int NRp,
                                                             const int *__restrict__ cls_real, double inv_s_real,
                                                             double inv_s_cplx, int d4, Format fmt, void *K1h, void *K1l,
                                                             void *K2h, void *K2l, void *K3h, void *K3l, void *K4h, void *K4l,
                                                             long long ldk, double *__restrict__ BR) {
    __shared__ double ts[4][32][33];
    const long long r0 = (long long)blockIdx.y * 32;
    const int i0 = blockIdx.x * 32;
    const double k4 = d4 ? 1.0 : 0.0;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const long long r = r0 + j;
        const int i = i0 + threadIdx.x;
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        if (r < rows && i < N) {
            const long long g = r / (2LL * NR);
            const long long rem = r - g * 2LL * NR;
            const bool imag = rem >= NR;
            const bool real_cls = cls_real[g] != 0;
            if (!(imag && real_cls)) {
                const long long o = r * ld;
                const double a = (double)H[o + i], b = (double)H[o + N + i], c = (double)Ch[o + i], d = (double)Ch[o + N + i];
                const double Ap = (double)HQ[o + i], Bp = (double)HQ[o + N + i], Cq = (double)Cp[o + i], Dq = (double)Cp[o + N + i];
                const double kk2 = -c / 3.0 + k4 * a / 8.0;
                v[0] = k4 * Ap / 8.0 - Dq / 3.0;
                v[1] = kk2;
                v[2] = -Ap / 6.0;
                v[3] = -a / 6.0;
                const double br = 0.5 * (-d / 3.0 + k4 * b / 4.0) * Ap + kk2 * Bp - a / 6.0 * Cq - b / 3.0 * Dq;
                BR[r * N + i] = br * (real_cls ? inv_s_real : inv_s_cplx);
            } else {
                BR[r * N + i] = 0.0;
            }
            if constexpr (!TRANS) {
                store_split(fmt, K1h, K1l, r * ldk + i, v[0]);
                store_split(fmt, K2h, K2l, r * ldk + i, v[1]);
                store_split(fmt, K3h, K3l, r * ldk + i, v[2]);
                store_split(fmt, K4h, K4l, r * ldk + i, v[3]);
            }
        }
        if constexpr (TRANS) {
#pragma unroll
            for (int q = 0; q < 4; ++q) ts[q][j][threadIdx.x] = v[q];
        }
    }
    if constexpr (TRANS) {
        __syncthreads();
        void *hs[4] = {K1h, K2h, K3h, K4h}, *ls[4] = {K1l, K2l, K3l, K4l};
        for (int j = threadIdx.y; j < 32; j += blockDim.y) {
            const int i = i0 + j;
            const long long r = r0 + threadIdx.x;
            if (i >= N || r >= rows) continue;
            const long long g = r / (2LL * NR);
            const long long rem = r - g * 2LL * NR;
            const long long comp = rem / NR, jj = rem - comp * NR;
            if (comp == 1 && cls_real[g]) continue;   // stays zero
            const long long col = g * 2LL * NRp + comp * NRp + jj;
#pragma unroll
            for (int q = 0; q < 4; ++q) store_split(fmt, hs[q], ls[q], (long long)i * ldk + col, ts[q][threadIdx.x][j]);
        }
    }
}

template <typename T>
__global__ void vjp_recon_pairs_kernel(int N, long long P, int Kq, const T *__restrict__ VbarQ, const int *__restrict__ col0,
                                       const int *__restrict__ col1, const double *__restrict__ pc0, const double *__restrict__ pc1,
                                       const double *__restrict__ pre, T *__restrict__ Vbar, long long ldv) {
    for (long long i = blockIdx.y; i < N; i += gridDim.y) {
        const T *q = VbarQ + i * Kq;
        for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
            const int a = col0[p];
            double v = pc0[p] * (double)q[a] / pre[a];
            const double k1 = pc1[p];
            if (k1 != 0.0) {
                const int b = col1[p];
                v += k1 * (double)q[b] / pre[b];
            }
            Vbar[i * ldv + p] = (T)v;
        }
    }
}

template <typename T>
__global__ void vjp_recon_modes_kernel(int N, int n, int Kmq, const T *__restrict__ GQ, const T *__restrict__ YQ,
                                       const int *__restrict__ mode_col, const double *__restrict__ sign,
                                       const double *__restrict__ mre, T *__restrict__ gbar, T *__restrict__ ypart, long long ldg) {
    const long long total = (long long)N * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const long long i = idx / n;
        const int m = (int)(idx - i * n);
        const int c = mode_col[m];
        double g = 0.0, y = 0.0;
        if (c >= 0) {
            const double f = sign[c] / mre[c];
            g = f * (double)GQ[i * Kmq + c];
            y = f * (double)YQ[i * Kmq + c];
        }
        gbar[i * ldg + m] = (T)g;
        ypart[i * ldg + m] = (T)y;
    }
}

}  // namespace

int freq_build_mode_rows(const FreqTables &t, const double *A, const double *B, int n, long long Nc, Format fmt, void *hi,
                         void *lo, cudaStream_t st) {
    if (t.Kmq == 0) return 0;
    build_XGq_kernel<<<grid1(2 * Nc * t.Kmq), 256, 0, st>>>(A, B, n, Nc, t.Kmq, t.mc_mode, t.mc_sign, fmt, hi, lo);
    TD_CUDA(cudaGetLastError());
    return 0;
}

int freq_transpose_left(Format fmt, const void *L, int NR, int NRp, long long cols, void *out, cudaStream_t st) {
    if (!L || cols <= 0) return 0;
    TD_CHECK(NRp % 32 == 0 && NR <= NRp && 2LL * NRp / 32 <= 65535 && ceil_div(cols, 32) <= 2147483647LL, TDSCHA_EINVAL,
             "left-operand transpose of %d rows x %lld", NR, cols);
    const dim3 grid((unsigned)ceil_div(cols, 32), (unsigned)(2 * NRp / 32)), block(32, 8);
    if (fmt == FMT_BF16)
        transpose_left_kernel<uint16_t><<<grid, block, 0, st>>>(static_cast<const uint16_t *>(L), NR, NRp, cols, static_cast<uint16_t *>(out));
    else if (fmt == FMT_F64)
        transpose_left_kernel<double><<<grid, block, 0, st>>>(static_cast<const double *>(L), NR, NRp, cols, static_cast<double *>(out));
    else
        transpose_left_kernel<float><<<grid, block, 0, st>>>(static_cast<const float *>(L), NR, NRp, cols, static_cast<float *>(out));
    TD_CUDA(cudaGetLastError());
    return 0;
}

template <typename AccT>
int freq_vjp_coef(const FreqTables &t, int sub, const AccT *H, const AccT *Ch, const AccT *HQ, const AccT *Cp, long long ld,
                  int N, int NR, int NRp, int d4, bool trans, Format fmt, void *const *K_hi, void *const *K_lo, long long ldk,
                  double *BR, cudaStream_t st) {
    const long long rows = (long long)t.n_class * 2 * NR;
    TD_CHECK(ceil_div(rows, 32) <= 65535, TDSCHA_EINVAL, "VJP coefficient grid: %lld rows", rows);
    const dim3 grid((unsigned)ceil_div(N, 32), (unsigned)ceil_div(rows, 32)), block(32, 8);
    const double inv_r = 1.0 / (double)sub, inv_c = 2.0 / (double)sub;
    if (trans)
        vjp_coef_class_kernel<AccT, true><<<grid, block, 0, st>>>(H, Ch, HQ, Cp, ld, N, rows, NR, NRp, t.d_cls_real, inv_r, inv_c, d4,
                                                                  fmt, K_hi[0], K_lo[0], K_hi[1], K_lo[1], K_hi[2], K_lo[2], K_hi[3],
                                                                  K_lo[3], ldk, BR);
    else
        vjp_coef_class_kernel<AccT, false><<<grid, block, 0, st>>>(H, Ch, HQ, Cp, ld, N, rows, NR, NRp, t.d_cls_real, inv_r, inv_c,
                                                                   d4, fmt, K_hi[0], K_lo[0], K_hi[1], K_lo[1], K_hi[2], K_lo[2],
                                                                   K_hi[3], K_lo[3], ldk, BR);
    TD_CUDA(cudaGetLastError());
    return 0;
}

template <typename T>
int freq_vjp_reconstruct(const FreqTables &t, int N, int n, long long P, const T *VbarQ, const T *GQ, const T *YQ, T *Vbar,
                         long long ldv, T *gbar, T *ypart, long long ldg, cudaStream_t st) {
    vjp_recon_pairs_kernel<T><<<grid_rows(P, N), 256, 0, st>>>(N, P, t.Kq, VbarQ, t.pp_col0, t.pp_col1, t.pp_c0, t.pp_c1, t.pc_re,
                                                               Vbar, ldv);
    vjp_recon_modes_kernel<T><<<grid1((long long)N * n), 256, 0, st>>>(N, n, t.Kmq, GQ, YQ, t.mode_col, t.mc_sign, t.mc_re, gbar,
                                                                         ypart, ldg);
    TD_CUDA(cudaGetLastError());
    return 0;
}

template int freq_vjp_coef<float>(const FreqTables &, int, const float *, const float *, const float *, const float *, long long,
                                  int, int, int, int, bool, Format, void *const *, void *const *, long long, double *,
                                  cudaStream_t);
template int freq_vjp_coef<double>(const FreqTables &, int, const double *, const double *, const double *, const double *,
                                   long long, int, int, int, int, bool, Format, void *const *, void *const *, long long, double *,
                                   cudaStream_t);
template int freq_vjp_reconstruct<float>(const FreqTables &, int, int, long long, const float *, const float *, const float *,
                                         float *, long long, float *, float *, long long, cudaStream_t);
template int freq_vjp_reconstruct<double>(const FreqTables &, int, int, long long, const double *, const double *, const double *,
                                          double *, long long, double *, double *, long long, cudaStream_t);

}  // namespace tdscha

// ================================================================================================
// Configuration chunks over a resident row-major class operand
// ================================================================================================
namespace tdscha {
namespace {

// out (cols x ldo) column q = in row (q < Nc ? ra + q : rb + q - Nc) for q < 2Nc, zero after; 32 x 32
// tiles through shared memory
template <typename T>
__global__ void transpose_two_ranges_kernel(const T *__restrict__ in, long long cols, long long ra, long long rb, long long Nc,
                                            T *__restrict__ out, long long ldo) {
    __shared__ T tile[32][33];
    const long long c0 = (long long)blockIdx.x * 32, q0 = (long long)blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const long long q = q0 + j, c = c0 + threadIdx.x;
        T v = T(0);
        if (q < 2 * Nc && c < cols) v = in[(q < Nc ? ra + q : rb + q - Nc) * cols + c];
        tile[j][threadIdx.x] = v;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const long long c = c0 + j, q = q0 + threadIdx.x;
        if (c < cols && q < ldo) out[c * ldo + q] = tile[threadIdx.x][j];
    }
}

template <typename T>
int transpose_two_ranges(const void *in, long long cols, long long ra, long long rb, long long Nc, void *out, long long ldo,
                         cudaStream_t st) {
    TD_CHECK(ldo % 32 == 0 && ldo / 32 <= 65535, TDSCHA_EINVAL, "chunk transpose: %lld columns", ldo);
    const dim3 grid((unsigned)ceil_div(cols, 32), (unsigned)(ldo / 32)), block(32, 8);
    transpose_two_ranges_kernel<T><<<grid, block, 0, st>>>(static_cast<const T *>(in), cols, ra, rb, Nc, static_cast<T *>(out), ldo);
    TD_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace

size_t freq_resident_rows_bytes(const FreqTables &t, long long N, Format fmt, bool lo) {
    return (size_t)2 * N * (t.Kq + t.Kmq) * format_bytes(fmt) * (lo ? 2 : 1) + 8 * 256;
}

size_t freq_chunk_cols_bytes(const FreqTables &t, long long Nc, Format fmt, bool lo) {
    const long long N2pc = round_up(2 * Nc, 64);
    return (size_t)N2pc * (t.Kq + t.Kmq) * format_bytes(fmt) * (lo ? 2 : 1) + 8 * 256;
}

int freq_build_rows(const FreqTables &t, const double *X, const double *G, const double *XGT, long long ldT, int n, long long N,
                    Format fmt, bool lo, void *buf, FreqOps &o, cudaStream_t st) {
    TD_CHECK(fmt == FMT_BF16 || fmt == FMT_TF32, TDSCHA_EINVAL, "resident class rows need a split format");
    const size_t es = format_bytes(fmt);
    const long long N2p = round_up(2 * N, 64);
    uint8_t *b = static_cast<uint8_t *>(buf);
    size_t off = 0;
    auto take = [&](long long count) { void *p = b + off; off += ((size_t)count * es + 255) / 256 * 256; return p; };
    o = FreqOps();
    o.V_hi = take(2 * N * t.Kq);
    o.XG_hi = take(2 * N * t.Kmq);
    if (lo) {
        o.V_lo = take(2 * N * t.Kq);
        o.XG_lo = take(2 * N * t.Kmq);
    }
    if (fmt == FMT_BF16)
        TD_TRY(build_Vq_cols<uint16_t>(t, XGT, ldT, n, N, N2p, fmt, o.V_hi, o.V_lo, nullptr, nullptr, st));
    else
        TD_TRY(build_Vq_cols<float>(t, XGT, ldT, n, N, N2p, fmt, o.V_hi, o.V_lo, nullptr, nullptr, st));
    if (t.Kmq > 0)
        build_XGq_kernel<<<grid1(2 * N * t.Kmq), 256, 0, st>>>(X, G, n, N, t.Kmq, t.mc_mode, t.mc_sign, fmt, o.XG_hi, o.XG_lo);
    TD_CUDA(cudaGetLastError());
    o.built = true;
    o.has_lo = lo;
    o.bytes = off;
    return 0;
}

int freq_build_chunk_cols(const FreqTables &t, const FreqOps &rows, long long N, long long c0, long long Nc, const double *Y,
                          const double *Xt, int n, Format fmt, bool lo, void *buf, FreqOps &o, cudaStream_t st) {
    const size_t es = format_bytes(fmt);
    const long long N2pc = round_up(2 * Nc, 64);
    uint8_t *b = static_cast<uint8_t *>(buf);
    size_t off = 0;
    auto take = [&](long long count) { void *p = b + off; off += ((size_t)count * es + 255) / 256 * 256; return p; };
    o = FreqOps();
    o.V_hi = rows.V_hi;
    o.V_lo = rows.V_lo;
    o.XG_hi = rows.XG_hi;
    o.XG_lo = rows.XG_lo;
    o.VT_hi = take((long long)t.Kq * N2pc);
    o.YX_hi = take((long long)t.Kmq * N2pc);
    if (lo) {
        o.VT_lo = take((long long)t.Kq * N2pc);
        o.YX_lo = take((long long)t.Kmq * N2pc);
    }
    for (int part = 0; part < (lo ? 2 : 1); ++part) {
        const void *src = part ? rows.V_lo : rows.V_hi;
        void *dst = part ? o.VT_lo : o.VT_hi;
        if (fmt == FMT_BF16) TD_TRY(transpose_two_ranges<uint16_t>(src, t.Kq, c0, N + c0, Nc, dst, N2pc, st));
        else TD_TRY(transpose_two_ranges<float>(src, t.Kq, c0, N + c0, Nc, dst, N2pc, st));
    }
    if (t.Kmq > 0)
        build_YXq_kernel<<<grid1((long long)t.Kmq * N2pc), 256, 0, st>>>(Y + c0 * n, Xt + c0 * n, n, Nc, N2pc, t.Kmq, t.mc_mode,
                                                                           t.mc_sign, fmt, o.YX_hi, o.YX_lo);
    TD_CUDA(cudaGetLastError());
    o.built = true;
    o.has_lo = lo;
    o.bytes = off;
    return 0;
}

}  // namespace tdscha
