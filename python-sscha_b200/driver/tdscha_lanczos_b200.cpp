// tdscha_lanczos_b200.cpp -- the B200 counterpart of the reference's stand-alone Lanczos program
// (CModules/main.cpp, CModules/Lanczos.cpp: tdscha-lanczos.x).
//
//   tdscha_lanczos_b200 <rootname> [--precision fp64|tf32|bf16x3|tf32x3|bf16] [--device K] [--quiet]
//
// Reads the input files that Lanczos.prepare_input_files writes (Modules/DynamicalLanczos.py:815-921):
// <root>.json, .X.dat, .Y.dat, .freqs, .rho, .psi, .ndegs, .blockid, .block<i>, .symsb<i>
// (Lanczos.cpp:47-269), runs the bi-conjugate Lanczos on the GPU through the library's C ABI
// (one batched apply of [L q, L^T p] and one recurrence launch per step) and writes the reference
// program's outputs (Lanczos.cpp:533-800): <root>.abc ("a\tb\tc" per step, a lone a on
// convergence), <root>.qbasis.out, <root>.pbasis.out (one vector per line), <root>.snorm.out.
// "restart": true with "step_done": k in the json resumes from those files, as the reference does.
//
// The operator follows the Python class (as every other entry point of this library): the shift
// adds shift * psi (the reference program adds the constant `shift` to every component,
// Lanczos.cpp:522-525), and the flag combinations on which the program and the Python class
// disagree are refused instead of silently differing: ignore_v3 without ignore_v4 (the program
// keeps the quartic term alone, Lanczos.cpp:420-437) and use_wigner (the program ignores it).
#include <cuda_runtime.h>

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "tdscha_b200.h"

using std::string;
using std::vector;

namespace {

// ---- a small JSON reader: objects, numbers, booleans, strings, null ----------------------------
struct JVal {
    enum Kind { NUL, BOOL, NUM, STR, OBJ, ARR } kind = NUL;
    bool b = false;
    double num = 0;
    string str;
    std::map<string, JVal> obj;
    vector<JVal> arr;
};

class JsonParser {
public:
    explicit JsonParser(const string &s) : s_(s) {}
    JVal parse() {
        JVal v = value();
        ws();
        if (i_ != s_.size()) fail("trailing characters");
        return v;
    }

private:
    const string &s_;
    size_t i_ = 0;
    [[noreturn]] void fail(const string &what) {
        throw std::runtime_error("json: " + what + " at offset " + std::to_string(i_));
    }
    void ws() {
        while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) ++i_;
    }
    bool eat(char c) {
        ws();
        if (i_ < s_.size() && s_[i_] == c) { ++i_; return true; }
        return false;
    }
    string str_lit() {
        if (!eat('"')) fail("expected string");
        string out;
        while (i_ < s_.size() && s_[i_] != '"') {
            if (s_[i_] == '\\' && i_ + 1 < s_.size()) { out += s_[i_ + 1]; i_ += 2; }
            else out += s_[i_++];
        }
        if (i_ >= s_.size()) fail("unterminated string");
        ++i_;
        return out;
    }
    JVal value() {
        ws();
        if (i_ >= s_.size()) fail("unexpected end");
        JVal v;
        const char c = s_[i_];
        if (c == '{') {
            ++i_;
            v.kind = JVal::OBJ;
            if (eat('}')) return v;
            do {
                string k = str_lit();
                if (!eat(':')) fail("expected ':'");
                v.obj[k] = value();
            } while (eat(','));
            if (!eat('}')) fail("expected '}'");
        } else if (c == '[') {
            ++i_;
            v.kind = JVal::ARR;
            if (eat(']')) return v;
            do { v.arr.push_back(value()); } while (eat(','));
            if (!eat(']')) fail("expected ']'");
        } else if (c == '"') {
            v.kind = JVal::STR;
            v.str = str_lit();
        } else if (s_.compare(i_, 4, "true") == 0) {
            v.kind = JVal::BOOL; v.b = true; i_ += 4;
        } else if (s_.compare(i_, 5, "false") == 0) {
            v.kind = JVal::BOOL; v.b = false; i_ += 5;
        } else if (s_.compare(i_, 4, "null") == 0) {
            i_ += 4;
        } else {
            char *end = nullptr;
            v.num = std::strtod(s_.c_str() + i_, &end);
            if (end == s_.c_str() + i_) fail("bad value");
            v.kind = JVal::NUM;
            i_ = (size_t)(end - s_.c_str());
        }
        return v;
    }
};

const JVal &child(const JVal &o, const string &k) {
    auto it = o.obj.find(k);
    if (o.kind != JVal::OBJ || it == o.obj.end()) throw std::runtime_error("json: missing key '" + k + "'");
    return it->second;
}
double num(const JVal &o, const string &k) { return child(o, k).num; }
bool flag(const JVal &o, const string &k) {
    const JVal &v = child(o, k);
    return v.kind == JVal::BOOL ? v.b : v.num != 0;
}
bool has(const JVal &o, const string &k) { return o.kind == JVal::OBJ && o.obj.count(k) > 0; }

// whitespace-separated numbers, exactly `count` of them
template <typename T>
vector<T> read_values(const string &path, size_t count) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    vector<T> out(count);
    for (size_t k = 0; k < count; ++k) {
        double v;
        if (!(f >> v)) throw std::runtime_error(path + ": expected " + std::to_string(count) + " values, found " + std::to_string(k));
        out[k] = (T)v;
    }
    return out;
}

void check(int rc, const char *what) {
    if (rc != TDSCHA_OK) throw std::runtime_error(string(what) + ": " + tdscha_last_error());
}
void check_cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(string(what) + ": " + cudaGetErrorString(e));
}

struct DevBuf {
    double *p = nullptr;
    explicit DevBuf(size_t n) { check_cuda(cudaMalloc(&p, n * sizeof(double)), "cudaMalloc"); }
    ~DevBuf() { if (p) cudaFree(p); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
};

int precision_code(const string &s) {
    if (s == "fp64") return TDSCHA_PREC_FP64;
    if (s == "tf32") return TDSCHA_PREC_TF32;
    if (s == "bf16x3") return TDSCHA_PREC_BF16X3;
    if (s == "tf32x3") return TDSCHA_PREC_TF32X3;
    if (s == "bf16") return TDSCHA_PREC_BF16;
    throw std::runtime_error("unknown precision '" + s + "'");
}

void usage() {
    std::cout << "LANCZOS CALCULATOR PROGRAM (B200)\n\nUsage:\n"
                 "  tdscha_lanczos_b200 <rootname> [--precision fp64|tf32|bf16x3|tf32x3|bf16] [--device K] [--quiet]\n\n"
                 "<rootname> is the name used by Lanczos.prepare_input_files to save the data.\n";
}

int run(int argc, char **argv) {
    if (argc < 2) { usage(); return EXIT_FAILURE; }
    string root = argv[1];
    int prec = TDSCHA_PREC_FP64, device = 0;
    bool quiet = false;
    for (int a = 2; a < argc; ++a) {
        string s = argv[a];
        if (s == "--precision" && a + 1 < argc) prec = precision_code(argv[++a]);
        else if (s == "--device" && a + 1 < argc) device = std::atoi(argv[++a]);
        else if (s == "--quiet") quiet = true;
        else { usage(); return EXIT_FAILURE; }
    }
    check_cuda(cudaSetDevice(device), "cudaSetDevice");

    // ---- input (Lanczos.cpp:47-269) ----
    std::ifstream jf(root + ".json");
    if (!jf) throw std::runtime_error("cannot open " + root + ".json");
    std::stringstream ss;
    ss << jf.rdbuf();
    const JVal js = JsonParser(ss.str()).parse();
    const double T = num(js, "T");
    const int n_steps = (int)num(js, "n_steps");
    const bool ignore_v2 = flag(js, "ignore_v2"), ignore_v3 = flag(js, "ignore_v3"), ignore_v4 = flag(js, "ignore_v4");
    bool restart = false;
    int step_done = 0;
    if (has(js, "restart")) {
        restart = flag(js, "restart");
        step_done = (int)num(js, "step_done");
    }
    if (step_done >= n_steps) throw std::runtime_error("n_steps must be greater than step_done");
    if (has(js, "use_wigner") && flag(js, "use_wigner"))
        throw std::runtime_error("use_wigner: this program runs the standard representation only, as tdscha-lanczos.x "
                                 "does; run the Wigner chain through the Python class");
    if (ignore_v3 && !ignore_v4)
        throw std::runtime_error("ignore_v3 without ignore_v4 (quartic term alone) is not available: the Python class "
                                 "and this library drop the whole anharmonic part with ignore_v3");
    const JVal &data = child(js, "data");
    const int N = (int)num(data, "n_configs"), n = (int)num(data, "n_modes");
    const int n_syms = (int)num(data, "n_syms"), n_blocks = (int)num(data, "n_blocks");
    const bool reverse_L = flag(data, "reverse");
    const double shift = num(data, "shift");
    const long long n_psi = (long long)n + (long long)n * (n + 1);

    vector<int> n_deg = read_values<int>(root + ".ndegs", n_blocks);
    vector<double> w = read_values<double>(root + ".freqs", n);
    vector<double> rho = read_values<double>(root + ".rho", N);
    vector<double> psi = read_values<double>(root + ".psi", n_psi);
    vector<double> X = read_values<double>(root + ".X.dat", (size_t)N * n);
    vector<double> Y = read_values<double>(root + ".Y.dat", (size_t)N * n);
    vector<int> blocks_ids = read_values<int>(root + ".blockid", n);
    vector<vector<int>> deg(n_blocks);
    vector<vector<double>> syms(n_blocks);
    vector<const int *> deg_p(n_blocks);
    vector<const double *> sym_p(n_blocks);
    for (int b = 0; b < n_blocks; ++b) {
        deg[b] = read_values<int>(root + ".block" + std::to_string(b), n_deg[b]);
        syms[b] = read_values<double>(root + ".symsb" + std::to_string(b), (size_t)n_syms * n_deg[b] * n_deg[b]);
        deg_p[b] = deg[b].data();
        sym_p[b] = syms[b].data();
    }

    // ---- history (restart) or first vector ----
    vector<double> a, bcf, ccf, snorm;
    vector<double> q_prev(n_psi, 0.0), p_prev(n_psi, 0.0), q(n_psi), p(n_psi);
    if (restart) {
        vector<double> abc = read_values<double>(root + ".abc", (size_t)3 * step_done);
        for (int k = 0; k < step_done; ++k) {
            a.push_back(abc[3 * k]);
            bcf.push_back(abc[3 * k + 1]);
            ccf.push_back(abc[3 * k + 2]);
        }
        vector<double> Q = read_values<double>(root + ".qbasis.out", (size_t)n_psi * (step_done + 1));
        vector<double> P = read_values<double>(root + ".pbasis.out", (size_t)n_psi * (step_done + 1));
        snorm = read_values<double>(root + ".snorm.out", step_done + 1);
        std::copy(Q.end() - n_psi, Q.end(), q.begin());
        std::copy(P.end() - n_psi, P.end(), p.begin());
        if (step_done >= 1) {
            std::copy(Q.end() - 2 * n_psi, Q.end() - n_psi, q_prev.begin());
            std::copy(P.end() - 2 * n_psi, P.end() - n_psi, p_prev.begin());
        }
    } else {
        double nrm = 0;
        for (double v : psi) nrm += v * v;
        nrm = std::sqrt(nrm);
        if (!(nrm > 0)) throw std::runtime_error("the starting vector (.psi) is zero");
        for (long long j = 0; j < n_psi; ++j) q[j] = p[j] = psi[j] / nrm;
        snorm.push_back(1.0);
    }

    tdscha_ensemble *ens = nullptr;
    check(tdscha_ensemble_create(X.data(), Y.data(), w.data(), rho.data(), N, n, T, n_syms, n_blocks, n_deg.data(),
                                 deg_p.data(), sym_p.data(), blocks_ids.data(), &ens),
          "tdscha_ensemble_create");
    std::unique_ptr<tdscha_ensemble, int (*)(tdscha_ensemble *)> ens_guard(ens, tdscha_ensemble_destroy);
    tdscha_apply_opts opts{0, (int)ignore_v2, (int)ignore_v3, (int)ignore_v4, (int)reverse_L, shift};

    DevBuf vec(2 * n_psi), out(2 * n_psi), dq(n_psi), dp(n_psi), dqp(n_psi), dpp(n_psi), dqn(n_psi), dpn(n_psi),
        sc_in(6), sc_out(4);
    auto up = [&](double *dst, const vector<double> &src) {
        check_cuda(cudaMemcpy(dst, src.data(), src.size() * sizeof(double), cudaMemcpyHostToDevice), "upload");
    };
    up(dq.p, q);
    up(dp.p, p);
    up(dqp.p, q_prev);
    up(dpp.p, p_prev);

    // ---- output files (Lanczos.cpp:573-621) ----
    const auto mode = restart ? (std::ios::out | std::ios::app) : std::ios::out;
    std::ofstream f_abc(root + ".abc", mode), f_q(root + ".qbasis.out", mode), f_p(root + ".pbasis.out", mode),
        f_s(root + ".snorm.out", mode);
    if (!f_abc || !f_q || !f_p || !f_s) throw std::runtime_error("cannot open the output files of " + root);
    for (auto *f : {&f_abc, &f_q, &f_p, &f_s}) *f << std::scientific << std::setprecision(16);
    auto write_vec = [](std::ofstream &f, const vector<double> &v) {
        for (double x : v) f << x << " ";
        f << std::endl;
    };
    if (!restart) {
        write_vec(f_q, q);
        write_vec(f_p, p);
        f_s << snorm[0] << std::endl;
    }

    const int transpose[2] = {0, 1};
    bool converged = false;
    double a_last = 0;
    vector<double> hq(n_psi), hp(n_psi);
    for (int step = (int)a.size(); step < n_steps; ++step) {
        check_cuda(cudaMemcpy(vec.p, dq.p, n_psi * sizeof(double), cudaMemcpyDeviceToDevice), "copy q");
        check_cuda(cudaMemcpy(vec.p + n_psi, dp.p, n_psi * sizeof(double), cudaMemcpyDeviceToDevice), "copy p");
        check(tdscha_apply_full_L_device(ens, 2, vec.p, transpose, &opts, prec, out.p, nullptr), "apply_full_L");
        const double sc[6] = {ccf.empty() ? 0.0 : ccf.back(), bcf.empty() ? 0.0 : bcf.back(), snorm.back(),
                              snorm.size() > 1 ? snorm[snorm.size() - 2] : 0.0, ccf.size() > 1 ? ccf[ccf.size() - 2] : 1.0,
                              (double)a.size()};
        check_cuda(cudaMemcpy(sc_in.p, sc, sizeof(sc), cudaMemcpyHostToDevice), "upload step scalars");
        check(tdscha_lanczos_step_device(1, n_psi, out.p, out.p + n_psi, dq.p, dp.p, dqp.p, dpp.p, sc_in.p, nullptr,
                                         dqn.p, dpn.p, sc_out.p, nullptr),
              "lanczos_step");
        double so[4];
        check_cuda(cudaMemcpy(so, sc_out.p, sizeof(so), cudaMemcpyDeviceToHost), "download step scalars");
        const double ak = so[0], bk = so[1], ck = so[2], snew = so[3];
        if (std::isnan(ak)) throw std::runtime_error("invalid value encountered during the Lanczos");
        a.push_back(ak);
        a_last = ak;
        if (std::fabs(bk) < 1e-12 || std::fabs(ck) < 1e-12) { converged = true; break; }
        bcf.push_back(bk);
        ccf.push_back(ck);
        snorm.push_back(snew);
        std::swap(dqp.p, dq.p);
        std::swap(dpp.p, dp.p);
        std::swap(dq.p, dqn.p);
        std::swap(dp.p, dpn.p);
        check_cuda(cudaMemcpy(hq.data(), dq.p, n_psi * sizeof(double), cudaMemcpyDeviceToHost), "download q");
        check_cuda(cudaMemcpy(hp.data(), dp.p, n_psi * sizeof(double), cudaMemcpyDeviceToHost), "download p");
        if (!quiet)
            std::cout << "a_" << step << " = " << std::scientific << std::setprecision(16) << ak << "\nb_" << step << " = "
                      << bk << "\nc_" << step << " = " << ck << "\n" << std::endl;
        f_abc << ak << "\t" << bk << "\t" << ck << std::endl;
        f_s << snew << std::endl;
        write_vec(f_q, hq);
        write_vec(f_p, hp);
    }
    if (converged) {
        if (!quiet) std::cout << "  Converged.\n The last a coefficient is " << std::scientific << std::setprecision(16) << a_last << std::endl;
        f_abc << a_last << std::endl;
    }
    if (!quiet) std::cout << "I'm done with the calculation!" << std::endl;
    return EXIT_SUCCESS;
}

}  // namespace

int main(int argc, char **argv) {
    try {
        return run(argc, argv);
    } catch (const std::exception &e) {
        std::cerr << "tdscha_lanczos_b200: " << e.what() << std::endl;
        return EXIT_FAILURE;
    }
}
