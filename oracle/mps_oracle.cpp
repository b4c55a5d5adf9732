// ORACLE — test infrastructure only.
//
// A CPU, FP64, single-threaded restatement of wqc-core's gate-by-gate MPS
// executor (the `cpu` backend of src/tn/mps.rs with src/tn/svd_guard.rs and
// src/tn/gates.rs).  It is the checker for the cuda backend and the timed CPU
// baseline; nothing in the product links or calls it.
//
// Parity pins: the reference crate cannot be built here (Rust toolchain and
// its git sibling wqc-stark-engine are absent), so this file is pinned to the
// reference's own unit tests and published values (see tests/test_oracle_*.py).
//
// Third-party arithmetic the reference calls and that is not vendored under
// the reference tree: nalgebra 0.33.3 (Cargo.lock:1106) complex SVD
// (`svd(true, true)`, Golub-Kahan bidiagonalisation + implicit-shift QR) and
// Householder QR (`qr().q()`).  They are restated below from the published
// algorithms (Golub & Reinsch 1970; Golub & Van Loan, Matrix Computations,
// 4th ed., Alg. 5.4.2 and 8.6.2); results agree with nalgebra up to the gauge
// of singular vectors, which no output of the MPS path depends on.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "../include/wqc_types.h"

namespace {

using cd = std::complex<double>;

thread_local std::string g_last_error;

struct EngineError : std::runtime_error {
    explicit EngineError(const std::string& m) : std::runtime_error(m) {}
};

// ---------------------------------------------------------------------------
// Dense column-major complex matrix.
// ---------------------------------------------------------------------------
struct CMat {
    int rows = 0, cols = 0;
    std::vector<cd> a;  // column-major
    CMat() = default;
    CMat(int r, int c) : rows(r), cols(c), a(size_t(r) * c, cd(0, 0)) {}
    cd& operator()(int i, int j) { return a[size_t(j) * rows + i]; }
    const cd& operator()(int i, int j) const { return a[size_t(j) * rows + i]; }
    cd* col(int j) { return &a[size_t(j) * rows]; }
    const cd* col(int j) const { return &a[size_t(j) * rows]; }
    static CMat identity(int n) {
        CMat m(n, n);
        for (int i = 0; i < n; ++i) m(i, i) = 1.0;
        return m;
    }
    CMat adjoint() const {
        CMat t(cols, rows);
        for (int j = 0; j < cols; ++j)
            for (int i = 0; i < rows; ++i) t(j, i) = std::conj((*this)(i, j));
        return t;
    }
    CMat transpose() const {
        CMat t(cols, rows);
        for (int j = 0; j < cols; ++j)
            for (int i = 0; i < rows; ++i) t(j, i) = (*this)(i, j);
        return t;
    }
};

CMat matmul(const CMat& x, const CMat& y) {
    CMat c(x.rows, y.cols);
    for (int j = 0; j < y.cols; ++j) {
        cd* cj = c.col(j);
        for (int k = 0; k < x.cols; ++k) {
            const cd ykj = y(k, j);
            if (ykj == cd(0, 0)) continue;
            const cd* xk = x.col(k);
            for (int i = 0; i < x.rows; ++i) cj[i] += xk[i] * ykj;
        }
    }
    return c;
}

struct Svd {
    CMat u;               // rows x k
    std::vector<double> s;  // k, descending
    CMat vt;              // k x cols (V^H)
    bool ok = true;
};

// ---------------------------------------------------------------------------
// Householder reflector (LAPACK zlarfg convention).  Given alpha = x[0] and the
// tail x[1:], returns tau and beta (real) and scales the tail into v[1:], with
// v[0] = 1 implicit, such that H^H x = beta e1 for H = I - tau v v^H.
// ---------------------------------------------------------------------------
void householder(cd& alpha, cd* tail, int len, cd& tau) {
    double xnorm2 = 0;
    for (int i = 0; i < len; ++i) xnorm2 += std::norm(tail[i]);
    const double ar = alpha.real(), ai = alpha.imag();
    if (xnorm2 == 0.0 && ai == 0.0) {
        tau = 0.0;
        return;
    }
    double beta = std::sqrt(ar * ar + ai * ai + xnorm2);
    if (ar >= 0) beta = -beta;
    tau = cd((beta - ar) / beta, -ai / beta);
    const cd scale = 1.0 / (alpha - beta);
    for (int i = 0; i < len; ++i) tail[i] *= scale;
    alpha = beta;
}

// Apply H = I - tau v v^H (v[0] = 1 implicit, v[1:] = vt) from the left to
// columns [c0, c1) of m restricted to rows [r0, rows): m <- H m.
void apply_left(CMat& m, int r0, const cd* vt, cd tau, int c0, int c1) {
    if (tau == cd(0, 0)) return;
    const int len = m.rows - r0;
    for (int j = c0; j < c1; ++j) {
        cd* cj = m.col(j) + r0;
        cd w = cj[0];
        for (int i = 1; i < len; ++i) w += std::conj(vt[i - 1]) * cj[i];
        w *= tau;
        cj[0] -= w;
        for (int i = 1; i < len; ++i) cj[i] -= vt[i - 1] * w;
    }
}

// ---------------------------------------------------------------------------
// Golub-Kahan-Reinsch SVD (the algorithm family of nalgebra's `svd`).
// Householder bidiagonalisation to a real bidiagonal, then implicit-shift QR
// sweeps with Givens rotations accumulated into U and V.
// ---------------------------------------------------------------------------
Svd gk_svd_tall(const CMat& a_in) {
    const int m = a_in.rows, n = a_in.cols;  // m >= n
    CMat a = a_in;
    std::vector<cd> tau_l(n, 0.0), tau_r(n, 0.0);
    std::vector<double> d(n, 0.0), e(n, 0.0);  // e[i] couples i and i+1
    for (int k = 0; k < n; ++k) {
        // Left reflector: zero a[k+1:, k], leave a real diagonal.
        cd alpha = a(k, k);
        householder(alpha, a.col(k) + k + 1, m - k - 1, tau_l[k]);
        a(k, k) = alpha;
        // Apply H^H to the trailing columns (H^H = I - conj(tau) v v^H).
        apply_left(a, k, a.col(k) + k + 1, std::conj(tau_l[k]), k + 1, n);
        d[k] = alpha.real();
        if (k + 1 < n) {
            // Right reflector on the row a[k, k+1:]: reflect x = conj(row)^T.
            const int len = n - k - 1;
            std::vector<cd> x(len);
            for (int j = 0; j < len; ++j) x[j] = std::conj(a(k, k + 1 + j));
            cd al = x[0];
            householder(al, x.data() + 1, len - 1, tau_r[k]);
            // Row becomes (beta, 0, ...): store beta, keep v tail in the row.
            a(k, k + 1) = al;
            for (int j = 1; j < len; ++j) a(k, k + 1 + j) = x[j];
            e[k] = al.real();
            // Apply H from the right to rows k+1..m-1, columns k+1..n-1:
            // A <- A H = A - tau (A v) v^H.
            const cd t = tau_r[k];
            if (t != cd(0, 0)) {
                for (int i = k + 1; i < m; ++i) {
                    cd w = a(i, k + 1);
                    for (int j = 1; j < len; ++j) w += a(i, k + 1 + j) * x[j];
                    w *= t;
                    a(i, k + 1) -= w;
                    for (int j = 1; j < len; ++j) a(i, k + 1 + j) -= w * std::conj(x[j]);
                }
            }
        }
    }
    // Accumulate U = H_0 ... H_{n-1} [I; 0] (m x n), backward.
    CMat u(m, n);
    for (int i = 0; i < n; ++i) u(i, i) = 1.0;
    for (int k = n - 1; k >= 0; --k) apply_left(u, k, a.col(k) + k + 1, tau_l[k], k, n);
    // Accumulate V = G_0 ... G_{n-2} (n x n), backward.  The reflector of row
    // k acts on coordinates k+1..n-1 with vector (1, x[1:]) where x[j] is
    // stored in a(k, k+1+j).
    CMat v = CMat::identity(n);
    for (int k = n - 2; k >= 0; --k) {
        const cd t = tau_r[k];
        if (t == cd(0, 0)) continue;
        const int len = n - k - 1;
        for (int j = k + 1; j < n; ++j) {
            cd* cj = v.col(j) + k + 1;
            cd w = cj[0];
            for (int i = 1; i < len; ++i) w += std::conj(a(k, k + 1 + i)) * cj[i];
            w *= t;
            cj[0] -= w;
            for (int i = 1; i < len; ++i) cj[i] -= a(k, k + 1 + i) * w;
        }
    }

    // Bidiagonal implicit-shift QR (Golub & Reinsch).  rv[i] = e[i-1].
    std::vector<double> w = d, rv(n, 0.0);
    for (int i = 1; i < n; ++i) rv[i] = e[i - 1];
    double anorm = 0;
    for (int i = 0; i < n; ++i) anorm = std::max(anorm, std::fabs(w[i]) + std::fabs(rv[i]));
    auto rot_cols = [](CMat& mat, int p, int q, double c, double s) {
        cd* xp = mat.col(p);
        cd* xq = mat.col(q);
        for (int r = 0; r < mat.rows; ++r) {
            const cd y = xp[r], z = xq[r];
            xp[r] = y * c + z * s;
            xq[r] = z * c - y * s;
        }
    };
    bool converged_all = true;
    for (int k = n - 1; k >= 0; --k) {
        for (int its = 0;; ++its) {
            bool cancel = true;
            int l = k, nm = 0;
            for (; l >= 0; --l) {
                nm = l - 1;
                if (std::fabs(rv[l]) + anorm == anorm) {
                    cancel = false;
                    break;
                }
                if (std::fabs(w[nm]) + anorm == anorm) break;
            }
            if (cancel) {
                double c = 0.0, s = 1.0;
                for (int i = l; i <= k; ++i) {
                    const double f = s * rv[i];
                    rv[i] = c * rv[i];
                    if (std::fabs(f) + anorm == anorm) break;
                    const double g = w[i];
                    double h = std::hypot(f, g);
                    w[i] = h;
                    h = 1.0 / h;
                    c = g * h;
                    s = -f * h;
                    rot_cols(u, nm, i, c, s);
                }
            }
            double z = w[k];
            if (l == k) {
                if (z < 0.0) {
                    w[k] = -z;
                    for (int r = 0; r < n; ++r) v(r, k) = -v(r, k);
                }
                break;
            }
            if (its >= 75) {
                converged_all = false;
                break;
            }
            double x = w[l];
            nm = k - 1;
            double y = w[nm];
            double g = rv[nm];
            double h = rv[k];
            double f = ((y - z) * (y + z) + (g - h) * (g + h)) / (2.0 * h * y);
            g = std::hypot(f, 1.0);
            f = ((x - z) * (x + z) + h * ((y / (f + std::copysign(g, f))) - h)) / x;
            double c = 1.0, s = 1.0;
            for (int j = l; j <= nm; ++j) {
                const int i = j + 1;
                g = rv[i];
                y = w[i];
                h = s * g;
                g = c * g;
                z = std::hypot(f, h);
                rv[j] = z;
                c = f / z;
                s = h / z;
                f = x * c + g * s;
                g = g * c - x * s;
                h = y * s;
                y *= c;
                rot_cols(v, j, i, c, s);
                z = std::hypot(f, h);
                w[j] = z;
                if (z != 0.0) {
                    z = 1.0 / z;
                    c = f * z;
                    s = h * z;
                }
                f = c * g + s * y;
                x = c * y - s * g;
                rot_cols(u, j, i, c, s);
            }
            rv[l] = 0.0;
            rv[k] = f;
            w[k] = x;
        }
    }
    // Sort descending (stable on ties).
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return w[x] > w[y]; });
    Svd out;
    out.ok = converged_all;
    out.u = CMat(m, n);
    out.vt = CMat(n, n);
    out.s.resize(n);
    for (int t = 0; t < n; ++t) {
        const int j = order[t];
        out.s[t] = w[j];
        std::copy(u.col(j), u.col(j) + m, out.u.col(t));
        for (int c = 0; c < n; ++c) out.vt(t, c) = std::conj(v(c, j));
    }
    return out;
}

Svd gk_svd(const CMat& a) {
    if (a.rows >= a.cols) return gk_svd_tall(a);
    // A^H = U' S V'^H  =>  A = V' S U'^H.
    Svd t = gk_svd_tall(a.adjoint());
    Svd out;
    out.ok = t.ok;
    out.s = t.s;
    out.u = t.vt.adjoint();
    out.vt = t.u.adjoint();
    return out;
}

// ---------------------------------------------------------------------------
// src/tn/svd_guard.rs
// ---------------------------------------------------------------------------
constexpr double SINGULAR_CUTOFF = 1e-12;   // svd_guard.rs:12
constexpr double CHI_REL_GAP = 1e-3;        // svd_guard.rs:15
constexpr double CUTOFF_ABS_BAND = 1e-10;   // svd_guard.rs:18
constexpr double SVD_CHECK_TOL = 1e-9;      // svd_guard.rs:234

// svd_guard.rs:25-35
int retained_chi(const std::vector<double>& v, int max_bond, int rows, int cols) {
    if (v.empty() || max_bond == 0 || rows == 0 || cols == 0) return 0;
    int rank = 0;
    for (double s : v)
        if (s > SINGULAR_CUTOFF) ++rank;
    rank = std::max(rank, 1);
    return std::min(std::min(rank, max_bond), std::min(rows, cols));
}

// svd_guard.rs:40-55 (circle method)
std::vector<uint32_t> jacobi_pairs(int cols) {
    std::vector<int> players(cols);
    std::iota(players.begin(), players.end(), 0);
    std::vector<uint32_t> out;
    for (int step = 0; step + 1 < cols; ++step) {
        for (int i = 0; i < cols / 2; ++i) {
            out.push_back(uint32_t(players[i]));
            out.push_back(uint32_t(players[cols - 1 - i]));
        }
        const int last = players.back();
        players.pop_back();
        players.insert(players.begin() + 1, last);
    }
    return out;
}

// svd_guard.rs:58-76
bool needs_f64_fallback(const std::vector<double>& v, int chi) {
    for (double s : v)
        if (!std::isfinite(s) || s < 0.0) return true;
    for (double s : v)
        if (s > 0.0 && std::fabs(s - SINGULAR_CUTOFF) <= CUTOFF_ABS_BAND) return true;
    if (chi > 0 && chi < int(v.size())) {
        const double kept = v[chi - 1], dropped = v[chi];
        const double scale = std::max(std::max(kept, dropped), 1e-30);
        if (std::fabs(kept - dropped) / scale < CHI_REL_GAP) return true;
    }
    return false;
}

// svd_guard.rs:146-229: one-sided Hestenes Jacobi, rephase then real rotation.
Svd jacobi_svd(const CMat& a) {
    if (a.rows < a.cols) {
        Svd t = jacobi_svd(a.adjoint());
        Svd out;
        out.s = t.s;
        out.u = t.vt.adjoint();
        out.vt = t.u.adjoint();
        return out;
    }
    const int m = a.rows, n = a.cols;
    CMat w = a;
    CMat v = CMat::identity(n);
    for (int sweep = 0; sweep < 80; ++sweep) {
        bool rotated = false;
        for (int p = 0; p < n; ++p) {
            for (int q = p + 1; q < n; ++q) {
                double alpha = 0, beta = 0;
                cd gamma = 0;
                const cd* wp = w.col(p);
                const cd* wq = w.col(q);
                for (int r = 0; r < m; ++r) alpha += std::norm(wp[r]);
                for (int r = 0; r < m; ++r) beta += std::norm(wq[r]);
                for (int r = 0; r < m; ++r) gamma += std::conj(wp[r]) * wq[r];
                const double g = std::abs(gamma);
                if (g <= 1e-15 * std::sqrt(alpha * beta) || g == 0.0) continue;
                rotated = true;
                const cd phase = gamma / g;
                const double zeta = (beta - alpha) / (2.0 * g);
                const double t = std::copysign(1.0, zeta) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / std::sqrt(1.0 + t * t);
                const double s = c * t;
                for (CMat* mat : {&w, &v}) {
                    cd* xp = mat->col(p);
                    cd* xqc = mat->col(q);
                    for (int r = 0; r < mat->rows; ++r) {
                        const cd xpv = xp[r];
                        const cd xq = xqc[r] * std::conj(phase);
                        xp[r] = xpv * c - xq * s;
                        xqc[r] = (xpv * s + xq * c) * phase;
                    }
                }
            }
        }
        if (!rotated) break;
    }
    std::vector<std::pair<double, int>> order(n);
    for (int j = 0; j < n; ++j) {
        double s2 = 0;
        for (int r = 0; r < m; ++r) s2 += std::norm(w(r, j));
        order[j] = {std::sqrt(s2), j};
    }
    std::stable_sort(order.begin(), order.end(),
                     [](const std::pair<double, int>& x, const std::pair<double, int>& y) { return x.first > y.first; });
    Svd out;
    out.u = CMat(m, n);
    out.vt = CMat(n, n);
    out.s.resize(n);
    for (int k = 0; k < n; ++k) {
        const double sigma = order[k].first;
        const int j = order[k].second;
        out.s[k] = sigma;
        if (sigma > 0.0)
            for (int r = 0; r < m; ++r) out.u(r, k) = w(r, j) / sigma;
        for (int r = 0; r < n; ++r) out.vt(k, r) = std::conj(v(r, j));
    }
    return out;
}

// svd_guard.rs:242-283
bool svd_reproduces(const CMat& a, const Svd& svd) {
    const auto& s = svd.s;
    for (size_t i = 0; i < s.size(); ++i) {
        if (!std::isfinite(s[i]) || s[i] < 0.0) return false;
        if (i + 1 < s.size() && s[i] < s[i + 1]) return false;
    }
    double fro2 = 0;
    for (const cd& c : a.a) fro2 += std::norm(c);
    double s2 = 0;
    for (double x : s) s2 += x * x;
    const double scale = std::max(std::sqrt(fro2), 2.2250738585072014e-308);
    if (std::fabs(s2 - fro2) > SVD_CHECK_TOL * std::max(fro2, 2.2250738585072014e-308) + 1e-28) return false;
    const int k = int(s.size());
    if (svd.u.cols < k || svd.vt.rows < k || svd.u.rows != a.rows || svd.vt.cols != a.cols) return false;
    for (int probe = 0; probe < 2; ++probe) {
        std::vector<cd> x(a.cols);
        for (int j = 0; j < a.cols; ++j) {
            const double t = (double(j) + 1.0) * (0.754877666 + double(probe) * 0.56984029);
            x[j] = cd(std::sin(t), std::cos(t));
        }
        std::vector<cd> direct(a.rows, 0.0), inner(k, 0.0), rebuilt(a.rows, 0.0);
        for (int j = 0; j < a.cols; ++j)
            for (int i = 0; i < a.rows; ++i) direct[i] += a(i, j) * x[j];
        for (int r = 0; r < k; ++r) {
            cd acc = 0;
            for (int j = 0; j < a.cols; ++j) acc += svd.vt(r, j) * x[j];
            inner[r] = acc * s[r];
        }
        for (int r = 0; r < k; ++r)
            for (int i = 0; i < a.rows; ++i) rebuilt[i] += svd.u(i, r) * inner[r];
        double xn = 0, err = 0;
        for (const cd& c : x) xn += std::norm(c);
        xn = std::sqrt(xn);
        for (int i = 0; i < a.rows; ++i) err += std::norm(direct[i] - rebuilt[i]);
        err = std::sqrt(err);
        if (err > SVD_CHECK_TOL * scale * xn + 1e-14) return false;
    }
    return true;
}

int g_svd_retries = 0, g_svd_jacobi = 0;
// 0: Golub-Kahan primary (the reference's nalgebra family); 1: the Jacobi of
// svd_guard.rs as primary.  Only used to measure how sensitive a workload is
// to the choice of a correct FP64 SVD.
int g_primary_svd = 0;

// svd_guard.rs:91-139.  `route` reports 0 = primary, 1 = transpose, 2 = Jacobi.
Svd checked_svd(CMat mat, int* route = nullptr) {
    double fro2 = 0;
    for (const cd& c : mat.a) fro2 += std::norm(c);
    const double dust = std::sqrt(fro2) * 1e-14;
    for (cd& c : mat.a)
        if (std::abs(c) < dust) c = 0.0;
    Svd svd = g_primary_svd == 1 ? jacobi_svd(mat) : gk_svd(mat);
    if (svd.ok && svd_reproduces(mat, svd)) {
        if (route) *route = 0;
        return svd;
    }
    ++g_svd_retries;
    if (std::getenv("WQC_ORACLE_DEBUG")) {
        std::fprintf(stderr, "oracle svd: primary rejected on %dx%d (converged=%d):", mat.rows, mat.cols, int(svd.ok));
        for (double x : svd.s) std::fprintf(stderr, " %.17g", x);
        std::fprintf(stderr, "\n");
    }
    Svd t = gk_svd(mat.transpose());
    Svd flipped;
    flipped.s = t.s;
    flipped.u = t.vt.transpose();
    flipped.vt = t.u.transpose();
    if (t.ok && svd_reproduces(mat, flipped)) {
        if (route) *route = 1;
        return flipped;
    }
    ++g_svd_jacobi;
    Svd j = jacobi_svd(mat);
    if (svd_reproduces(mat, j)) {
        if (route) *route = 2;
        return j;
    }
    throw EngineError("SVD of a " + std::to_string(mat.rows) + "x" + std::to_string(mat.cols) +
                      " matrix failed its check");
}

// ---------------------------------------------------------------------------
// src/tn/gates.rs
// ---------------------------------------------------------------------------
struct Mat2 {
    cd u[2][2];
};
struct Mat4 {
    cd u[2][2][2][2];  // [c_out][t_out][c_in][t_in]
};

Mat2 unary_matrix(int kind, double theta) {
    const cd z(0, 0), o(1, 0), i(0, 1);
    Mat2 m{};
    switch (kind) {
        case WQC_GATE_H: {
            const double k = 1.0 / std::sqrt(2.0);
            m = {{{k, k}, {k, -k}}};
            break;
        }
        case WQC_GATE_X: m = {{{z, o}, {o, z}}}; break;
        case WQC_GATE_Y: m = {{{z, -i}, {i, z}}}; break;
        case WQC_GATE_Z: m = {{{o, z}, {z, -o}}}; break;
        case WQC_GATE_S: m = {{{o, z}, {z, i}}}; break;
        case WQC_GATE_T: {
            const double r = 0.70710678118654752440;  // FRAC_1_SQRT_2
            m = {{{o, z}, {z, cd(r, r)}}};
            break;
        }
        case WQC_GATE_RX: {
            const double s = std::sin(theta / 2.0), c = std::cos(theta / 2.0);
            m = {{{cd(c, 0), cd(0, -s)}, {cd(0, -s), cd(c, 0)}}};
            break;
        }
        case WQC_GATE_RY: {
            const double s = std::sin(theta / 2.0), c = std::cos(theta / 2.0);
            m = {{{cd(c, 0), cd(-s, 0)}, {cd(s, 0), cd(c, 0)}}};
            break;
        }
        case WQC_GATE_RZ: {
            const double s = std::sin(theta / 2.0), c = std::cos(theta / 2.0);
            m = {{{cd(c, -s), z}, {z, cd(c, s)}}};
            break;
        }
        default: throw EngineError("not a unary gate");
    }
    return m;
}

Mat2 tdg_matrix() {  // mps.rs:1173-1180
    const double r = 0.70710678118654752440;
    return Mat2{{{1.0, 0.0}, {0.0, cd(r, -r)}}};
}

Mat4 cnot_matrix() {
    Mat4 m{};
    m.u[0][0][0][0] = 1.0;
    m.u[0][1][0][1] = 1.0;
    m.u[1][0][1][1] = 1.0;
    m.u[1][1][1][0] = 1.0;
    return m;
}
Mat4 cz_matrix() {
    Mat4 m{};
    m.u[0][0][0][0] = 1.0;
    m.u[0][1][0][1] = 1.0;
    m.u[1][0][1][0] = 1.0;
    m.u[1][1][1][1] = -1.0;
    return m;
}
Mat4 swap_matrix() {
    Mat4 m{};
    m.u[0][0][0][0] = 1.0;
    m.u[0][1][1][0] = 1.0;
    m.u[1][0][0][1] = 1.0;
    m.u[1][1][1][1] = 1.0;
    return m;
}

Mat2 adjoint_mat2(const Mat2& u) {  // mps.rs:1203-1208
    Mat2 o;
    o.u[0][0] = std::conj(u.u[0][0]);
    o.u[0][1] = std::conj(u.u[1][0]);
    o.u[1][0] = std::conj(u.u[0][1]);
    o.u[1][1] = std::conj(u.u[1][1]);
    return o;
}
Mat4 adjoint_mat4(const Mat4& u) {  // mps.rs:1210-1223
    Mat4 o;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 2; ++c)
                for (int d = 0; d < 2; ++d) o.u[a][b][c][d] = std::conj(u.u[c][d][a][b]);
    return o;
}

// ---------------------------------------------------------------------------
// src/tn/mps.rs
// ---------------------------------------------------------------------------
struct Site {
    int l = 1, r = 1;
    std::vector<cd> a;  // [l][2][r]
    cd& at(int x, int s, int y) { return a[(size_t(x) * 2 + s) * r + y]; }
    const cd& at(int x, int s, int y) const { return a[(size_t(x) * 2 + s) * r + y]; }
};

constexpr int RSVD_MIN_SIDE = 160;   // mps.rs:794
constexpr int RSVD_OVERSAMPLE = 16;  // mps.rs:795

bool rsvd_worth(int rows, int cols, int ell) {  // mps.rs:929-935
    const unsigned __int128 f = (unsigned __int128)rows * cols * ell;
    const unsigned __int128 side = RSVD_MIN_SIDE;
    return f >= side * side * side;
}

uint64_t mix_seed(uint64_t rows, uint64_t cols, uint64_t ell) {  // mps.rs:1116-1122
    return (rows * 0x9E37ULL + cols) * 0x9E37ULL + ell;
}

// mps.rs:1103-1114 (row-major cols x ell)
std::vector<cd> rademacher(int cols, int ell, uint64_t salt) {
    uint64_t state = salt | 1ULL;
    const double scale = 1.0 / std::sqrt(double(cols));
    std::vector<cd> omega;
    omega.reserve(size_t(cols) * ell);
    for (size_t i = 0; i < size_t(cols) * ell; ++i) {
        state = state * 6364136223846793005ULL + 1ULL;
        const double re = (state & 0x100) == 0 ? scale : -scale;
        const double im = (state & 0x200) == 0 ? scale : -scale;
        omega.emplace_back(re, im);
    }
    return omega;
}

// Thin Q of a Householder QR (mps.rs:1091-1101 via nalgebra `qr().q()`).
CMat thin_q(const CMat& y) {
    const int m = y.rows, n = y.cols;
    const int k = std::min(m, n);
    CMat a = y;
    std::vector<cd> tau(k, 0.0);
    for (int j = 0; j < k; ++j) {
        cd alpha = a(j, j);
        householder(alpha, a.col(j) + j + 1, m - j - 1, tau[j]);
        a(j, j) = alpha;
        apply_left(a, j, a.col(j) + j + 1, std::conj(tau[j]), j + 1, n);
    }
    CMat q(m, k);
    for (int i = 0; i < k; ++i) q(i, i) = 1.0;
    for (int j = k - 1; j >= 0; --j) apply_left(q, j, a.col(j) + j + 1, tau[j], j, k);
    return q;
}

struct SplitOut {
    Site left, right;
    wqc_split_info info{};
};

// mps.rs:1124-1171 with the split record added.
void truncated_svd_split(const CMat& mat, int max_bond, int dl, int dr, bool reject, SplitOut& out) {
    const int rows = mat.rows, cols = mat.cols;
    Svd svd = checked_svd(mat);
    const int chi = retained_chi(svd.s, max_bond, rows, cols);
    if (reject) {
        for (size_t i = chi; i < svd.s.size(); ++i)
            if (svd.s[i] > SINGULAR_CUTOFF) throw EngineError("mps bond exceeded chi");
    }
    double disc = 0;
    for (size_t i = chi; i < svd.s.size(); ++i) disc += svd.s[i] * svd.s[i];
    out.left.l = dl;
    out.left.r = chi;
    out.left.a.assign(size_t(dl) * 2 * chi, 0.0);
    out.right.l = chi;
    out.right.r = dr;
    out.right.a.assign(size_t(chi) * 2 * dr, 0.0);
    for (int m = 0; m < chi; ++m) {
        const double s = std::sqrt(svd.s[m]);
        for (int l = 0; l < dl; ++l)
            for (int p = 0; p < 2; ++p) out.left.at(l, p, m) = svd.u(l * 2 + p, m) * s;
        for (int r = 0; r < dr; ++r)
            for (int t = 0; t < 2; ++t) out.right.at(m, t, r) = svd.vt(m, t * dr + r) * s;
    }
    out.info.chi = chi;
    out.info.discarded_weight = disc;
}

// mps.rs:983-1053.  Returns false when the range finder is rejected.
bool rsvd_sites(const CMat& mat, int ell, int dl, int dr, int max_bond, SplitOut& out) {
    const int rows = mat.rows, cols = mat.cols;
    const std::vector<cd> om = rademacher(cols, ell, mix_seed(rows, cols, ell));
    CMat omega(cols, ell);
    for (int r = 0; r < cols; ++r)
        for (int c = 0; c < ell; ++c) omega(r, c) = om[size_t(r) * ell + c];
    const CMat y0 = matmul(mat, omega);
    const CMat ah = mat.adjoint();
    const CMat z = matmul(ah, y0);
    const CMat y = matmul(mat, z);
    const CMat q = thin_q(y);
    const CMat b = matmul(q.adjoint(), mat);
    Svd svd;
    try {
        svd = checked_svd(b);
    } catch (const EngineError&) {
        return false;
    }
    std::vector<double> values = svd.s;
    for (double& s : values)
        if (s < SINGULAR_CUTOFF * 1e-2) s = 0.0;
    const int chi = retained_chi(values, max_bond, rows, cols);
    if (chi == 0 || needs_f64_fallback(values, chi)) return false;
    double disc = 0;
    for (size_t i = chi; i < values.size(); ++i) disc += values[i] * values[i];
    out.left.l = dl;
    out.left.r = chi;
    out.left.a.assign(size_t(dl) * 2 * chi, 0.0);
    out.right.l = chi;
    out.right.r = dr;
    out.right.a.assign(size_t(chi) * 2 * dr, 0.0);
    for (int mode = 0; mode < chi; ++mode) {
        const double scale = std::sqrt(svd.s[mode]);
        for (int r = 0; r < rows; ++r) {
            cd acc = 0;
            for (int t = 0; t < ell; ++t) acc += q(r, t) * svd.u(t, mode);
            out.left.at(r / 2, r % 2, mode) = acc * scale;
        }
        for (int c = 0; c < cols; ++c) out.right.at(mode, c / dr, c % dr) = svd.vt(mode, c) * scale;
    }
    out.info.chi = chi;
    out.info.discarded_weight = disc;
    return true;
}

// theta[a][s][t][b] flattened; mps.rs:1190-1199 / 955-964 matrix view.
CMat theta_matrix(const std::vector<cd>& theta, int dl, int dr) {
    const int rows = 2 * dl, cols = 2 * dr;
    CMat m(rows, cols);
    for (int a = 0; a < dl; ++a)
        for (int s = 0; s < 2; ++s)
            for (int t = 0; t < 2; ++t)
                for (int b = 0; b < dr; ++b) m(a * 2 + s, t * dr + b) = theta[((size_t(a) * 2 + s) * 2 + t) * dr + b];
    return m;
}

// mps.rs:937-981
// `exact_only` is the backend's exact split rule (no range finder), used to
// compare large splits reproducibly; the reference rule is exact_only = false.
void split_theta(const std::vector<cd>& theta, int dl, int dr, int max_bond, bool reject, SplitOut& out,
                 bool exact_only = false) {
    const int rows = dl * 2, cols = 2 * dr;
    const CMat mat = theta_matrix(theta, dl, dr);
    out.info.rows = rows;
    out.info.cols = cols;
    out.info.ell = std::min(std::min(max_bond + RSVD_OVERSAMPLE, rows), cols);
    if (exact_only && !reject) {
        out.info.path = WQC_SPLIT_EXACT;
        truncated_svd_split(mat, max_bond, dl, dr, false, out);
        return;
    }
    if (reject) {
        out.info.path = WQC_SPLIT_EXACT;
        truncated_svd_split(mat, max_bond, dl, dr, true, out);
        return;
    }
    const int ell = out.info.ell;
    if (ell == 0 || ell >= std::min(rows, cols) || !rsvd_worth(rows, cols, ell)) {
        out.info.path = WQC_SPLIT_EXACT;
        truncated_svd_split(mat, max_bond, dl, dr, false, out);
        return;
    }
    if (rsvd_sites(mat, ell, dl, dr, max_bond, out)) {
        out.info.path = WQC_SPLIT_RSVD;
        return;
    }
    out.info.path = WQC_SPLIT_RSVD_FALLBACK;
    truncated_svd_split(mat, max_bond, dl, dr, false, out);
}

struct Mps {
    int n = 0;
    int max_bond = 0;
    bool reject_truncation = false;
    bool exact_only = false;
    std::vector<Site> sites;
    std::vector<wqc_split_info> records;

    Mps(int n_, int chi, bool reject) : n(n_), max_bond(chi), reject_truncation(reject) {
        if (n_ <= 0) throw EngineError("Invalid qubit count: " + std::to_string(n_) + ". Max limit is 40.");
        if (chi <= 0) throw EngineError("MPS max bond dimension must be > 0");
        sites.resize(n_);
        for (auto& s : sites) {
            s.l = s.r = 1;
            s.a.assign(2, 0.0);
            s.a[0] = 1.0;
        }
    }

    // mps.rs:333-351
    void apply_one_qubit(int q, const Mat2& u) {
        Site& s = sites.at(q);
        Site upd;
        upd.l = s.l;
        upd.r = s.r;
        upd.a.assign(s.a.size(), 0.0);
        for (int a = 0; a < s.l; ++a)
            for (int b = 0; b < s.r; ++b) {
                const cd v0 = s.at(a, 0, b), v1 = s.at(a, 1, b);
                upd.at(a, 0, b) = u.u[0][0] * v0 + u.u[0][1] * v1;
                upd.at(a, 1, b) = u.u[1][0] * v0 + u.u[1][1] * v1;
            }
        s = std::move(upd);
    }

    // mps.rs:484-514 / 812-831
    static std::vector<cd> merge(const Site& left, const Site& right) {
        const int dl = left.l, dr = right.r, bond = std::min(left.r, right.l);
        std::vector<cd> theta(size_t(dl) * 4 * dr, 0.0);
        for (int a = 0; a < dl; ++a)
            for (int b = 0; b < dr; ++b)
                for (int s = 0; s < 2; ++s)
                    for (int t = 0; t < 2; ++t) {
                        cd sum = 0;
                        for (int g = 0; g < bond; ++g) sum += left.at(a, s, g) * right.at(g, t, b);
                        theta[((size_t(a) * 2 + s) * 2 + t) * dr + b] = sum;
                    }
        return theta;
    }

    // mps.rs:833-866 (also the inline loop at 396-421)
    static std::vector<cd> apply_two_qubit_unitary(const std::vector<cd>& theta, int dl, int dr, const Mat4& u,
                                                   bool ctrl_is_first) {
        std::vector<cd> upd(theta.size(), 0.0);
        for (int a = 0; a < dl; ++a)
            for (int b = 0; b < dr; ++b)
                for (int so = 0; so < 2; ++so)
                    for (int to = 0; to < 2; ++to) {
                        cd sum = 0;
                        for (int si = 0; si < 2; ++si)
                            for (int ti = 0; ti < 2; ++ti) {
                                const int c_out = ctrl_is_first ? so : to, t_out = ctrl_is_first ? to : so;
                                const int c_in = ctrl_is_first ? si : ti, t_in = ctrl_is_first ? ti : si;
                                sum += u.u[c_out][t_out][c_in][t_in] * theta[((size_t(a) * 2 + si) * 2 + ti) * dr + b];
                            }
                        upd[((size_t(a) * 2 + so) * 2 + to) * dr + b] = sum;
                    }
        return upd;
    }

    void split_into(int p, const std::vector<cd>& updated, int dl, int dr) {
        SplitOut out;
        split_theta(updated, dl, dr, max_bond, reject_truncation, out, exact_only);
        out.info.left_site = p;
        sites[p] = std::move(out.left);
        sites[p + 1] = std::move(out.right);
        records.push_back(out.info);
    }

    // mps.rs:377-429
    void apply_two_qubit_at_positions(int p, int q, const Mat4& u, bool ctrl_is_first) {
        if (q != p + 1) throw EngineError("two-site apply needs adjacent positions");
        const Site left = sites.at(p), right = sites.at(q);
        const int dl = left.l, dr = right.r;
        const std::vector<cd> theta = merge(left, right);
        const std::vector<cd> upd = apply_two_qubit_unitary(theta, dl, dr, u, ctrl_is_first);
        split_into(p, upd, dl, dr);
    }

    void apply_swap_positions(int p, int q) { apply_two_qubit_at_positions(p, q, swap_matrix(), true); }

    // mps.rs:353-375
    void apply_two_qubit_gate(int ctrl, int tgt, const Mat4& u) {
        const int left = std::min(ctrl, tgt), right = std::max(ctrl, tgt);
        const int span = right - left;
        if (span > 1)
            for (int pos = right - 1; pos >= left + 1; --pos) apply_swap_positions(pos, pos + 1);
        apply_two_qubit_at_positions(left, left + 1, u, ctrl < tgt);
        if (span > 1)
            for (int pos = left + 1; pos < right; ++pos) apply_swap_positions(pos, pos + 1);
    }

    // mps.rs:657-677
    void apply_ccnot(int c1, int c2, int t) {
        const Mat2 tdg = tdg_matrix();
        const Mat2 h = unary_matrix(WQC_GATE_H, 0), tt = unary_matrix(WQC_GATE_T, 0);
        const Mat4 cx = cnot_matrix();
        apply_one_qubit(t, h);
        apply_two_qubit_gate(c2, t, cx);
        apply_one_qubit(t, tdg);
        apply_two_qubit_gate(c1, t, cx);
        apply_one_qubit(t, tt);
        apply_two_qubit_gate(c2, t, cx);
        apply_one_qubit(t, tdg);
        apply_two_qubit_gate(c1, t, cx);
        apply_one_qubit(t, tt);
        apply_one_qubit(t, h);
        apply_one_qubit(c2, tt);
        apply_two_qubit_gate(c1, c2, cx);
        apply_one_qubit(c1, tt);
        apply_one_qubit(c2, tdg);
        apply_two_qubit_gate(c1, c2, cx);
    }

    void check_qubit(int q) const {
        if (q < 0 || q >= n)
            throw EngineError("Qubit index " + std::to_string(q) + " out of bounds (limit: " + std::to_string(n) + ")");
    }

    // mps.rs:278-297
    void apply_gate(const wqc_gate& g) {
        switch (g.kind) {
            case WQC_GATE_H: case WQC_GATE_X: case WQC_GATE_Y: case WQC_GATE_Z: case WQC_GATE_S:
            case WQC_GATE_T: case WQC_GATE_RX: case WQC_GATE_RY: case WQC_GATE_RZ:
                check_qubit(g.q0);
                apply_one_qubit(g.q0, unary_matrix(g.kind, g.angle));
                break;
            case WQC_GATE_CNOT:
                check_qubit(g.q0); check_qubit(g.q1);
                apply_two_qubit_gate(g.q0, g.q1, cnot_matrix());
                break;
            case WQC_GATE_CZ:
                check_qubit(g.q0); check_qubit(g.q1);
                apply_two_qubit_gate(g.q0, g.q1, cz_matrix());
                break;
            case WQC_GATE_CCNOT:
                check_qubit(g.q0); check_qubit(g.q1); check_qubit(g.q2);
                apply_ccnot(g.q0, g.q1, g.q2);
                break;
            default: break;  // MEASURE / RESET / IF
        }
    }

    // mps.rs:301-331
    void apply_gate_adjoint(const wqc_gate& g) {
        switch (g.kind) {
            case WQC_GATE_MEASURE: case WQC_GATE_RESET: case WQC_GATE_IF:
                throw EngineError("time-split overlap does not apply measurement or reset");
            case WQC_GATE_CCNOT: apply_ccnot(g.q0, g.q1, g.q2); break;
            case WQC_GATE_CNOT: apply_two_qubit_gate(g.q0, g.q1, adjoint_mat4(cnot_matrix())); break;
            case WQC_GATE_CZ: apply_two_qubit_gate(g.q0, g.q1, adjoint_mat4(cz_matrix())); break;
            default: apply_one_qubit(g.q0, adjoint_mat2(unary_matrix(g.kind, g.angle))); break;
        }
    }

    // mps.rs:520-565: merge every job from the current sites, then split each.
    void apply_adjacent_disjoint_gates(const wqc_gate* gates, int count) {
        if (count < 2) {
            for (int i = 0; i < count; ++i) apply_gate(gates[i]);
            return;
        }
        struct Job {
            int p, q;
            bool cf;
            Mat4 u;
            std::vector<cd> theta;
            int dl, dr;
        };
        std::vector<Job> jobs;
        for (int i = 0; i < count; ++i) {
            const wqc_gate& g = gates[i];
            if (g.kind != WQC_GATE_CNOT && g.kind != WQC_GATE_CZ)
                throw EngineError("disjoint layer contains a gate that is not CNOT or CZ");
            const int c = g.q0, t = g.q1;
            Job j;
            j.p = std::min(c, t);
            j.q = std::max(c, t);
            j.cf = c < t;
            j.u = g.kind == WQC_GATE_CNOT ? cnot_matrix() : cz_matrix();
            j.dl = sites[j.p].l;
            j.dr = sites[j.q].r;
            j.theta = merge(sites[j.p], sites[j.q]);
            jobs.push_back(std::move(j));
        }
        for (Job& j : jobs) {
            const std::vector<cd> upd = apply_two_qubit_unitary(j.theta, j.dl, j.dr, j.u, j.cf);
            split_into(j.p, upd, j.dl, j.dr);
        }
    }

    // mps.rs:262-276
    cd amplitude_at_compact_zero() const {
        std::vector<cd> vec{1.0};
        for (const Site& s : sites) {
            std::vector<cd> next(s.r, 0.0);
            for (int a = 0; a < std::min<int>(s.l, int(vec.size())); ++a)
                for (int b = 0; b < s.r; ++b) next[b] += vec[a] * s.at(a, 0, b);
            vec.swap(next);
        }
        return vec.empty() ? cd(0, 0) : vec[0];
    }

    // mps.rs:700-740
    std::vector<cd> left_environment(int target) const {
        std::vector<cd> vec{1.0};
        for (int i = 0; i < target; ++i) {
            const Site& s = sites[i];
            std::vector<cd> next(s.r, 0.0);
            for (int a = 0; a < std::min<int>(s.l, int(vec.size())); ++a)
                for (int p = 0; p < 2; ++p)
                    for (int b = 0; b < s.r; ++b) next[b] += vec[a] * s.at(a, p, b);
            vec.swap(next);
        }
        return vec;
    }
    std::vector<cd> right_environment(int target) const {
        std::vector<cd> vec{1.0};
        if (target + 1 >= n) return vec;
        for (int i = n - 1; i > target; --i) {
            const Site& s = sites[i];
            std::vector<cd> next(s.l, 0.0);
            for (int b = 0; b < std::min<int>(s.r, int(vec.size())); ++b)
                for (int p = 0; p < 2; ++p)
                    for (int a = 0; a < s.l; ++a) next[a] += vec[b] * s.at(a, p, b);
            vec.swap(next);
        }
        return vec;
    }
    // mps.rs:679-693
    void site_amplitudes(int target, cd& a0, cd& a1) const {
        const auto le = left_environment(target);
        const auto re = right_environment(target);
        const Site& s = sites[target];
        a0 = a1 = 0.0;
        for (size_t l = 0; l < le.size(); ++l)
            for (int r = 0; r < s.r; ++r) {
                const cd rr = r < int(re.size()) ? re[r] : cd(1.0, 0.0);
                a0 += le[l] * s.at(int(l), 0, r) * rr;
                a1 += le[l] * s.at(int(l), 1, r) * rr;
            }
    }

    // mps.rs:742-780
    void fill_dense(int idx, int bond_in, uint64_t prefix, cd coeff, std::vector<cd>& st) const {
        if (idx == n) {
            st[prefix] += coeff;
            return;
        }
        const Site& s = sites[idx];
        if (bond_in >= s.l) return;
        for (int p = 0; p < 2; ++p)
            for (int b = 0; b < s.r; ++b) {
                const cd amp = s.at(bond_in, p, b);
                if (std::norm(amp) < 1e-30) continue;
                fill_dense(idx + 1, b, prefix | (uint64_t(p) << idx), coeff * amp, st);
            }
    }
    std::vector<cd> to_dense_state() const {
        std::vector<cd> st(size_t(1) << n, 0.0);
        fill_dense(0, 0, 0, 1.0, st);
        return st;
    }

    // mps.rs:215-260
    std::vector<cd> contract_to_statevector() const {
        if (n > 20) throw EngineError("full statevector projection requires qubit_count <= 20");
        std::vector<cd> state{1.0};
        for (int q = 0; q < n; ++q) {
            const Site& s = sites[q];
            const size_t prefix = size_t(1) << q;
            if (state.size() != size_t(s.l) * prefix)
                throw EngineError("MPS bond layout mismatch during statevector projection");
            std::vector<cd> next(size_t(s.r) * prefix * 2, 0.0);
            for (int a = 0; a < s.l; ++a)
                for (size_t bp = 0; bp < prefix; ++bp) {
                    const cd v = state[a * prefix + bp];
                    for (int p = 0; p < 2; ++p)
                        for (int b = 0; b < s.r; ++b) next[b * (prefix * 2) + bp + p * prefix] += v * s.at(a, p, b);
                }
            state.swap(next);
        }
        return state;
    }

    // Pauli-string expectation <psi|P|psi> by transfer matrices (an addition:
    // the reference densifies, expectation.rs:189-200).  Label character
    // n-1-q acts on qubit q (expectation.rs:98-132).
    cd pauli_expectation(const char* label) const {
        std::vector<cd> env{1.0};  // [l_ket][l_bra]
        int lk = 1;
        for (int q = 0; q < n; ++q) {
            const Site& s = sites[q];
            const char ch = label[n - 1 - q];
            cd P[2][2] = {{1, 0}, {0, 1}};  // P[s_out][s_in]
            if (ch == 'X') { P[0][0] = 0; P[0][1] = 1; P[1][0] = 1; P[1][1] = 0; }
            else if (ch == 'Y') { P[0][0] = 0; P[0][1] = cd(0, -1); P[1][0] = cd(0, 1); P[1][1] = 0; }
            else if (ch == 'Z') { P[1][1] = -1; }
            else if (ch != 'I') throw EngineError(std::string("invalid pauli character in label"));
            // tmp[l'][s][r] = sum_l env[l][l'] ket[l][s][r] (ket side), then
            // next[r][r'] = sum_{l',s,s'} conj(bra[l'][s'][r']) P[s'][s] tmp[l'][s][r]
            const int r = s.r;
            std::vector<cd> tmp(size_t(lk) * 2 * r, 0.0);
            for (int l = 0; l < lk; ++l)
                for (int lp = 0; lp < lk; ++lp) {
                    const cd e = env[size_t(l) * lk + lp];
                    if (e == cd(0, 0)) continue;
                    for (int p = 0; p < 2; ++p)
                        for (int b = 0; b < r; ++b) tmp[(size_t(lp) * 2 + p) * r + b] += e * s.at(l, p, b);
                }
            std::vector<cd> next(size_t(r) * r, 0.0);
            for (int lp = 0; lp < lk; ++lp)
                for (int so = 0; so < 2; ++so)
                    for (int si = 0; si < 2; ++si) {
                        const cd pv = P[so][si];
                        if (pv == cd(0, 0)) continue;
                        for (int b = 0; b < r; ++b) {
                            const cd t = pv * tmp[(size_t(lp) * 2 + si) * r + b];
                            for (int bp = 0; bp < r; ++bp) next[size_t(b) * r + bp] += std::conj(s.at(lp, so, bp)) * t;
                        }
                    }
            env.swap(next);
            lk = r;
        }
        return env[0];
    }
};

// trace.rs:203-262 helpers: the call sequence execute_with_trace_using makes.
bool is_rotation(int k) { return k == WQC_GATE_RX || k == WQC_GATE_RY || k == WQC_GATE_RZ; }

void execute_call_sequence(Mps& mps, const wqc_gate* gates, int count) {
    int i = 0;
    while (i < count) {
        const wqc_gate& g = gates[i];
        if (g.kind == WQC_GATE_MEASURE || g.kind == WQC_GATE_RESET || g.kind == WQC_GATE_IF) {
            ++i;
            continue;
        }
        if (g.kind == WQC_GATE_H) {  // trace.rs:78-97: every H of the run is applied
            int run = 1;
            while (i + run < count && gates[i + run].kind == WQC_GATE_H && gates[i + run].q0 == g.q0) ++run;
            for (int k = 0; k < run; ++k) mps.apply_gate(gates[i + k]);
            i += run;
            continue;
        }
        if (is_rotation(g.kind)) {  // trace.rs:99-129
            int run = 1;
            double sum = g.angle;
            while (i + run < count && gates[i + run].kind == g.kind && gates[i + run].q0 == g.q0) {
                sum += gates[i + run].angle;
                ++run;
            }
            const double tau = 6.283185307179586;
            double red = std::fmod(sum, tau);
            if (red < 0) red += tau;
            const bool identity = std::fabs(red) < 1e-9 || std::fabs(tau - red) < 1e-9;
            if (identity) {
                for (int k = 0; k < run; ++k) mps.apply_gate(gates[i + k]);
            } else {
                wqc_gate net = g;
                net.angle = sum;
                mps.apply_gate(net);
            }
            i += run;
            continue;
        }
        int layer = 0;  // trace.rs:135-154, adjacent_disjoint_len 243-262
        if (mps.n > 16) {
            std::vector<int> seen;
            int cnt = 0;
            for (int k = i; k < count; ++k) {
                const wqc_gate& h = gates[k];
                if (h.kind != WQC_GATE_CNOT && h.kind != WQC_GATE_CZ) break;
                if (std::abs(h.q0 - h.q1) != 1) break;
                const int lo = std::min(h.q0, h.q1), hi = std::max(h.q0, h.q1);
                if (std::find(seen.begin(), seen.end(), lo) != seen.end() ||
                    std::find(seen.begin(), seen.end(), hi) != seen.end())
                    break;
                seen.push_back(lo);
                seen.push_back(hi);
                ++cnt;
            }
            layer = cnt >= 2 ? cnt : 0;
        }
        if (layer >= 2) {
            mps.apply_adjacent_disjoint_gates(gates + i, layer);
            i += layer;
            continue;
        }
        mps.apply_gate(g);
        ++i;
    }
}

// mps.rs:1421-1474
cd overlap(const Mps& ket, const Mps& bra) {
    if (ket.n != bra.n) throw EngineError("Workspace/circuit qubit count mismatch");
    std::vector<cd> env{1.0};
    int kl = 1, bl = 1;
    for (int i = 0; i < ket.n; ++i) {
        const Site& kt = ket.sites[i];
        const Site& bt = bra.sites[i];
        if (kt.l != kl || bt.l != bl) throw EngineError("mps site shape does not match the overlap");
        const int env_dim = kt.r * bt.r;
        if (env_dim > 256) throw EngineError("mps overlap environment exceeds 256");
        std::vector<cd> next(env_dim, 0.0);
        for (int a = 0; a < kt.l; ++a)
            for (int b = 0; b < bt.l; ++b) {
                const cd coeff = env[size_t(a) * bl + b];
                if (std::norm(coeff) == 0.0) continue;
                for (int s = 0; s < 2; ++s)
                    for (int ar = 0; ar < kt.r; ++ar) {
                        const cd kv = coeff * kt.at(a, s, ar);
                        if (std::norm(kv) == 0.0) continue;
                        for (int bo = 0; bo < bt.r; ++bo) next[size_t(ar) * bt.r + bo] += kv * std::conj(bt.at(b, s, bo));
                    }
            }
        env.swap(next);
        kl = kt.r;
        bl = bt.r;
    }
    if (env.size() != 1) throw EngineError("mps overlap left an open bond");
    return env[0];
}

CMat from_rowmajor(int m, int n, const double* a) {
    CMat x(m, n);
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) x(i, j) = cd(a[2 * (size_t(i) * n + j)], a[2 * (size_t(i) * n + j) + 1]);
    return x;
}
void to_rowmajor(const CMat& x, double* out) {
    for (int i = 0; i < x.rows; ++i)
        for (int j = 0; j < x.cols; ++j) {
            out[2 * (size_t(i) * x.cols + j)] = x(i, j).real();
            out[2 * (size_t(i) * x.cols + j) + 1] = x(i, j).imag();
        }
}

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return 1;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI for the Python test harness and the CPU baseline timer.
// ---------------------------------------------------------------------------
extern "C" {

struct oracle_mps {
    Mps m;
};

const char* oracle_last_error(void) { return g_last_error.c_str(); }

int oracle_mps_create(int n, int chi, int reject_truncation, oracle_mps** out) {
    return guarded([&] { *out = new oracle_mps{Mps(n, chi, reject_truncation != 0)}; });
}
void oracle_mps_destroy(oracle_mps* m) { delete m; }

void oracle_mps_set_split_rule(oracle_mps* m, int rule) { m->m.exact_only = rule == 1; }
int oracle_mps_apply_gates(oracle_mps* m, const wqc_gate* g, int count) {
    return guarded([&] {
        for (int i = 0; i < count; ++i) m->m.apply_gate(g[i]);
    });
}
int oracle_mps_apply_call_sequence(oracle_mps* m, const wqc_gate* g, int count) {
    return guarded([&] { execute_call_sequence(m->m, g, count); });
}
int oracle_mps_apply_layer(oracle_mps* m, const wqc_gate* g, int count) {
    return guarded([&] { m->m.apply_adjacent_disjoint_gates(g, count); });
}
int oracle_mps_apply_1q(oracle_mps* m, int site, const double* u8) {
    return guarded([&] {
        Mat2 u;
        for (int i = 0; i < 4; ++i) u.u[i / 2][i % 2] = cd(u8[2 * i], u8[2 * i + 1]);
        m->m.check_qubit(site);
        m->m.apply_one_qubit(site, u);
    });
}
int oracle_mps_apply_2q(oracle_mps* m, int ctrl, int tgt, const double* u32) {
    return guarded([&] {
        Mat4 u;
        for (int i = 0; i < 16; ++i) u.u[i >> 3][(i >> 2) & 1][(i >> 1) & 1][i & 1] = cd(u32[2 * i], u32[2 * i + 1]);
        m->m.check_qubit(ctrl);
        m->m.check_qubit(tgt);
        m->m.apply_two_qubit_gate(ctrl, tgt, u);
    });
}
int oracle_mps_apply_2q_at(oracle_mps* m, int left_site, const double* u32, int ctrl_is_first) {
    return guarded([&] {
        Mat4 u;
        for (int i = 0; i < 16; ++i) u.u[i >> 3][(i >> 2) & 1][(i >> 1) & 1][i & 1] = cd(u32[2 * i], u32[2 * i + 1]);
        m->m.apply_two_qubit_at_positions(left_site, left_site + 1, u, ctrl_is_first != 0);
    });
}
int oracle_mps_amplitude_zero(oracle_mps* m, double* out) {
    const cd a = m->m.amplitude_at_compact_zero();
    out[0] = a.real();
    out[1] = a.imag();
    return 0;
}
int oracle_mps_site_amplitudes(oracle_mps* m, int target, double* out) {
    return guarded([&] {
        m->m.check_qubit(target);
        cd a0, a1;
        m->m.site_amplitudes(target, a0, a1);
        out[0] = a0.real(); out[1] = a0.imag(); out[2] = a1.real(); out[3] = a1.imag();
    });
}
int oracle_mps_bond_dims(oracle_mps* m, int* out) {
    for (int i = 0; i < m->m.n; ++i) out[i] = m->m.sites[i].r;
    return 0;
}
int oracle_mps_num_records(oracle_mps* m) { return int(m->m.records.size()); }
int oracle_mps_records(oracle_mps* m, wqc_split_info* out, int max) {
    const int k = std::min<int>(max, int(m->m.records.size()));
    std::memcpy(out, m->m.records.data(), sizeof(wqc_split_info) * k);
    return k;
}
int oracle_mps_dense(oracle_mps* m, double* out) {
    return guarded([&] {
        if (m->m.n > 24) throw EngineError("dense download is limited to 24 qubits");
        const auto st = m->m.to_dense_state();
        std::memcpy(out, st.data(), st.size() * sizeof(cd));
    });
}
int oracle_mps_statevector(oracle_mps* m, double* out) {
    return guarded([&] {
        const auto st = m->m.contract_to_statevector();
        std::memcpy(out, st.data(), st.size() * sizeof(cd));
    });
}
int oracle_mps_site(oracle_mps* m, int site, int* l, int* r, double* buf) {
    return guarded([&] {
        m->m.check_qubit(site);
        const Site& s = m->m.sites[site];
        *l = s.l;
        *r = s.r;
        if (buf) std::memcpy(buf, s.a.data(), s.a.size() * sizeof(cd));
    });
}
int oracle_mps_set_site(oracle_mps* m, int site, int l, int r, const double* buf) {
    return guarded([&] {
        m->m.check_qubit(site);
        Site s;
        s.l = l;
        s.r = r;
        s.a.assign(size_t(l) * 2 * r, 0.0);
        std::memcpy((void*)s.a.data(), buf, s.a.size() * sizeof(cd));
        m->m.sites[site] = std::move(s);
    });
}
int oracle_mps_expectation_pauli(oracle_mps* m, const char* labels, const double* coeffs, int nterms, double* out) {
    return guarded([&] {
        cd acc = 0;
        for (int t = 0; t < nterms; ++t) {
            const cd v = m->m.pauli_expectation(labels + size_t(t) * m->m.n);
            acc += cd(coeffs[2 * t], coeffs[2 * t + 1]) * v.real();
        }
        out[0] = acc.real();
        out[1] = acc.imag();
    });
}

// mps.rs:1241-1249 / 1358-1419: the bra runs the Gate-level adjoint sequence
// of the second half when every gate has one, else apply_gate_adjoint.
int oracle_time_split(int n, const wqc_gate* g, int count, int split, int max_bond, double* out) {
    return guarded([&] {
        if (split > count) throw EngineError("time-split index past the gate list");
        Mps ket(n, max_bond, true), bra(n, max_bond, true);
        for (int i = 0; i < split; ++i) ket.apply_gate(g[i]);
        std::vector<wqc_gate> seq;
        bool all = true;
        for (int i = count - 1; i >= split && all; --i) {
            wqc_gate h = g[i];
            switch (h.kind) {
                case WQC_GATE_RX: case WQC_GATE_RY: case WQC_GATE_RZ:
                    h.angle = -h.angle;
                    seq.push_back(h);
                    break;
                case WQC_GATE_S: {
                    wqc_gate z = h;
                    z.kind = WQC_GATE_Z;
                    seq.push_back(h);
                    seq.push_back(z);
                    break;
                }
                case WQC_GATE_T: {
                    wqc_gate z = h;
                    z.kind = WQC_GATE_Z;
                    seq.push_back(h);
                    seq.push_back(h);
                    seq.push_back(h);
                    seq.push_back(z);
                    break;
                }
                case WQC_GATE_MEASURE: case WQC_GATE_RESET: case WQC_GATE_IF: all = false; break;
                default: seq.push_back(h); break;
            }
        }
        if (all) {
            for (const wqc_gate& h : seq) bra.apply_gate(h);
        } else {
            for (int i = count - 1; i >= split; --i) bra.apply_gate_adjoint(g[i]);
        }
        const cd a = overlap(ket, bra);
        out[0] = a.real();
        out[1] = a.imag();
    });
}

// Standalone pieces for known-answer tests.  Matrices are row-major complex.
int oracle_checked_svd(int m, int n, const double* a, double* s, double* u, double* vt, int* route) {
    return guarded([&] {
        const Svd r = checked_svd(from_rowmajor(m, n, a), route);
        const int k = int(r.s.size());
        for (int i = 0; i < k; ++i) s[i] = r.s[i];
        if (u) to_rowmajor(r.u, u);
        if (vt) to_rowmajor(r.vt, vt);
    });
}
int oracle_gk_svd(int m, int n, const double* a, double* s, double* u, double* vt) {
    return guarded([&] {
        const Svd r = gk_svd(from_rowmajor(m, n, a));
        if (!r.ok) throw EngineError("no convergence");
        for (size_t i = 0; i < r.s.size(); ++i) s[i] = r.s[i];
        if (u) to_rowmajor(r.u, u);
        if (vt) to_rowmajor(r.vt, vt);
    });
}
int oracle_jacobi_svd(int m, int n, const double* a, double* s, double* u, double* vt) {
    return guarded([&] {
        const Svd r = jacobi_svd(from_rowmajor(m, n, a));
        for (size_t i = 0; i < r.s.size(); ++i) s[i] = r.s[i];
        if (u) to_rowmajor(r.u, u);
        if (vt) to_rowmajor(r.vt, vt);
    });
}
int oracle_thin_q(int m, int n, const double* a, double* q) {
    return guarded([&] { to_rowmajor(thin_q(from_rowmajor(m, n, a)), q); });
}
// mat is rows x cols row-major; left (dl,2,chi) and right (chi,2,dr) buffers
// must hold max_bond modes.  Returns 0 and *chi_out on acceptance, 2 when the
// range finder is rejected.
int oracle_rsvd_sites(int rows, int cols, int ell, int dl, int dr, int max_bond, const double* mat, int* chi_out,
                      double* left, double* right) {
    int rc = 0;
    const int g = guarded([&] {
        SplitOut out;
        if (!rsvd_sites(from_rowmajor(rows, cols, mat), ell, dl, dr, max_bond, out)) {
            rc = 2;
            return;
        }
        *chi_out = out.info.chi;
        std::memcpy(left, out.left.a.data(), out.left.a.size() * sizeof(cd));
        std::memcpy(right, out.right.a.data(), out.right.a.size() * sizeof(cd));
    });
    return g ? g : rc;
}
int oracle_retained_chi(const double* v, int len, int max_bond, int rows, int cols) {
    return retained_chi(std::vector<double>(v, v + len), max_bond, rows, cols);
}
int oracle_needs_f64_fallback(const double* v, int len, int chi) {
    return needs_f64_fallback(std::vector<double>(v, v + len), chi) ? 1 : 0;
}
int oracle_rsvd_worth(int rows, int cols, int ell) { return rsvd_worth(rows, cols, ell) ? 1 : 0; }
void oracle_jacobi_pairs(int cols, uint32_t* out) {
    const auto p = jacobi_pairs(cols);
    std::memcpy(out, p.data(), p.size() * sizeof(uint32_t));
}
uint64_t oracle_mix_seed(uint64_t rows, uint64_t cols, uint64_t ell) { return mix_seed(rows, cols, ell); }
void oracle_rademacher(int cols, int ell, uint64_t salt, double* out) {
    const auto o = rademacher(cols, ell, salt);
    std::memcpy(out, o.data(), o.size() * sizeof(cd));
}
void oracle_svd_counters(int* retries, int* jacobi) {
    *retries = g_svd_retries;
    *jacobi = g_svd_jacobi;
}
void oracle_set_primary_svd(int mode) { g_primary_svd = mode; }
// engine.rs:29-31: round half away from zero on the 1e-6 grid.
double oracle_snap(double x) { return std::round(x * 1e6) / 1e6; }
// mps.rs:27-32
uint64_t oracle_mps_workspace_bytes(uint64_t n, uint64_t chi) {
    const unsigned __int128 v = (unsigned __int128)n * chi * chi * 32;
    return v > ~uint64_t(0) ? ~uint64_t(0) : uint64_t(v);
}

}  // extern "C"
