// CPU restatement of the cable loss and of its discrete adjoint -- TEST
// INFRASTRUCTURE ONLY (the checker for the GPU cable kernels).
//
// Forward step: the monodomain step of oracle_tissue.cpp specialised to a 1D
// cable with the ODE step equal to the PDE step -- ComputeExceptVoltage by
// forward Euler (heart/src/odes/AbstractCardiacCell.cpp:90-105), GetIIonic
// after the ODE step (AbstractCardiacTissue::UpdateCaches), z = Am Cm V/dt -
// Am Iion - Istim(t+dt) (heart/src/solver/MonodomainSolver.cpp:92-101), and
// (Am Cm/dt M + K) V' = M z (MonodomainAssembler.cpp:43-66) by Jacobi CG with
// PETSc's KSPCG/KSPConvergedDefault stopping test.
//
// Gradient: the adjoint recursion, recomputing each checkpoint segment:
//   mu = A^{-1} lam ; dL/dsigma_e -= mu^T dK/dsigma_e V' ; lz = M mu ;
//   dL/dV += Am Cm/dt lz ; dL/dIion = -Am lz, then the reverse products of
//   GetIIonic and of the Euler step emitted with the cell model.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include <thread>

#include "oracle_internal.h"

// Dual numbers (value, derivative along one direction) for the tangent-linear
// run: the cell-model templates instantiated on Dual give exact directional
// derivatives of the same discrete step (branches follow the values).
namespace chb {
struct Dual {
    double v, d;
    constexpr Dual() : v(0.0), d(0.0) {}
    constexpr Dual(double x) : v(x), d(0.0) {}
    constexpr Dual(double x, double dx) : v(x), d(dx) {}
};
inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
inline Dual& operator+=(Dual& a, Dual b) { return a = a + b; }
inline Dual& operator-=(Dual& a, Dual b) { return a = a - b; }
inline Dual& operator*=(Dual& a, Dual b) { return a = a * b; }
inline Dual& operator/=(Dual& a, Dual b) { return a = a / b; }
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
inline Dual m_exp(Dual a) {
    const double e = std::exp(a.v);
    return Dual(e, e * a.d);
}
inline Dual m_log(Dual a) { return Dual(std::log(a.v), a.d / a.v); }
inline Dual m_sqrt(Dual a) {
    const double r = std::sqrt(a.v);
    return Dual(r, a.d / (2.0 * r));
}
inline Dual m_pow(Dual a, Dual b) {
    const double p = std::pow(a.v, b.v);
    double d = a.d != 0.0 ? b.v * std::pow(a.v, b.v - 1.0) * a.d : 0.0;
    if (b.d != 0.0) d += p * std::log(a.v) * b.d;
    return Dual(p, d);
}
inline Dual fabs(Dual a) { return a.v < 0.0 ? -a : a; }
inline Dual m_div(Dual a, Dual b) { return a / b; }
inline Dual m_divk(Dual x, Dual k, Dual) { return x / k; }
template <>
constexpr Dual singularity_offset<Dual>() { return Dual(1e-7); }
}  // namespace chb

namespace {

struct Tri {
    std::vector<double> d, o;   // diagonal, super-diagonal (o[i] couples i and i+1)
    void mul(const std::vector<double>& x, std::vector<double>& y) const {
        const int n = (int)d.size();
        for (int i = 0; i < n; ++i) {
            double acc = 0.0;
            if (i > 0) acc += o[i - 1] * x[i - 1];
            acc += d[i] * x[i];
            if (i < n - 1) acc += o[i] * x[i + 1];
            y[i] = acc;
        }
    }
};

double dot(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

// KSPSolve_CG (standard variant, preconditioned norm) with Jacobi; returns the
// iteration count or -1 at maxit.  b_norm: tolerance against ||B b||.
int cg(const Tri& A, const std::vector<double>& b, std::vector<double>& x, double rtol, int maxit, bool b_norm) {
    const int n = (int)b.size();
    std::vector<double> r(n), z(n), p(n), q(n), dinv(n);
    for (int i = 0; i < n; ++i) dinv[i] = 1.0 / A.d[i];
    A.mul(x, q);
    for (int i = 0; i < n; ++i) {
        r[i] = b[i] - q[i];
        z[i] = dinv[i] * r[i];
    }
    double dp = std::sqrt(dot(z, z));
    double rnorm0 = dp;
    if (b_norm) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += (dinv[i] * b[i]) * (dinv[i] * b[i]);
        rnorm0 = std::sqrt(s);
    }
    const double ttol = std::fmax(rtol * rnorm0, 1e-50);
    if (dp <= ttol) return 0;
    double beta = dot(z, r), betaold = 1.0;
    for (int it = 0; it < maxit; ++it) {
        if (beta == 0.0) return it;
        for (int i = 0; i < n; ++i) p[i] = it == 0 ? z[i] : z[i] + (beta / betaold) * p[i];
        A.mul(p, q);
        const double alpha = beta / dot(p, q);
        for (int i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
            z[i] = dinv[i] * r[i];
        }
        dp = std::sqrt(dot(z, z));
        if (dp <= ttol) return it + 1;
        betaold = beta;
        beta = dot(z, r);
    }
    return -1;
}

int node_region(int i, int n, int R) { return std::min(R - 1, i * R / n); }
int elem_region(int e, int n, int R) { return std::min(R - 1, e * R / (n - 1)); }

template <class M>
struct CableRun {
    static constexpr int S = M::kNumStates, P = M::kNumParams, W = P + 1;
    const orc_cable_config& c;
    const double* prm;
    int n, R, T;
    double ms, dur;
    Tri A, Mm;
    std::vector<double> z, b;

    CableRun(const orc_cable_config& cc, const double* p)
        : c(cc), prm(p), n(cc.n_nodes), R(cc.n_regions), T(cc.n_steps), z(cc.n_nodes), b(cc.n_nodes) {
        ms = c.am * c.cm / c.dt;
        dur = c.stim_dur + c.stim_dur * DBL_EPSILON;
        A.d.assign(n, 0.0);
        A.o.assign(n, 0.0);
        Mm.d.assign(n, 0.0);
        Mm.o.assign(n, 0.0);
        for (int e = 0; e < n - 1; ++e) {
            const double sig = c.sigma * prm[elem_region(e, n, R) * W + P];
            const double md = c.h * 2.0 / 6.0, mo = c.h / 6.0, k = sig / c.h;
            A.d[e] += ms * md + k;
            A.d[e + 1] += ms * md + k;
            A.o[e] = ms * mo - k;
            Mm.d[e] += md;
            Mm.d[e + 1] += md;
            Mm.o[e] = mo;
        }
    }
    double stim(int i, double t) const { return (i < c.n_stim && 0.0 <= t && t <= dur) ? c.stim_mag : 0.0; }
    const double* params_of(int i) const { return prm + node_region(i, n, R) * W; }

    // Step s: y (node-major, y[i*S] unused on entry) and V (V_s in, V_{s+1} out).
    bool step(int s, std::vector<double>& y, std::vector<double>& V) {
        const double t0 = s * c.dt, t1 = t0 + c.dt;
        for (int i = 0; i < n; ++i) {
            double* yi = &y[(size_t)i * S];
            yi[0] = V[i];
            const double* p = params_of(i);
            double dy[S];
            M::template rhs<double>(yi, stim(i, t0) / c.am, c.cm, p, dy);
            for (int k = 1; k < S; ++k) yi[k] += c.dt * dy[k];
            const double ii = M::template iionic<double>(yi, c.cm, p);
            z[i] = ms * V[i] + (-c.am * ii - stim(i, t1));
        }
        Mm.mul(z, b);
        return cg(A, b, V, c.rtol, c.max_iterations, true) >= 0;
    }
};

template <class M>
int run(const orc_cable_config& c, const double* prm, const int* probes, int np, const double* targets,
        double* loss_out, double* traces, double* grad) {
    using Run = CableRun<M>;
    constexpr int S = Run::S, P = Run::P, W = Run::W;
    const int n = c.n_nodes, R = c.n_regions, T = c.n_steps;
    if (n < 2 || R < 1 || T < 1) return -4;
    const int K = c.checkpoint_every > 0 ? c.checkpoint_every : T;
    const int n_ck = (T + K - 1) / K;
    if (grad && ((double)n * K * S > 4e7 || (double)n * n_ck * S > 4e7)) return -4;
    Run run_(c, prm);
    std::vector<double> y((size_t)n * S), V(n), ck;
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < S; ++k) y[(size_t)i * S + k] = M::kInitialStates[k];
    for (int i = 0; i < n; ++i) V[i] = y[(size_t)i * S];
    if (grad) ck.resize((size_t)n_ck * n * S);
    double loss = 0.0;
    for (int s = 0; s < T; ++s) {
        if (grad && s % K == 0) {
            double* dst = &ck[(size_t)(s / K) * n * S];
            for (int i = 0; i < n; ++i) {
                dst[(size_t)i * S] = V[i];
                for (int k = 1; k < S; ++k) dst[(size_t)i * S + k] = y[(size_t)i * S + k];
            }
        }
        if (!run_.step(s, y, V)) return -1;
        for (int k = 0; k < np; ++k) {
            if (traces) traces[(size_t)s * np + k] = V[probes[k]];
            if (targets) {
                const double d = V[probes[k]] - targets[(size_t)s * np + k];
                loss += d * d;
            }
        }
    }
    if (loss_out) *loss_out = loss / ((double)T * np);
    if (!grad) return 0;
    // adjoint sweep, one checkpoint segment at a time (recomputed, every state kept)
    for (int k = 0; k < R * W; ++k) grad[k] = 0.0;
    std::vector<double> lam(n, 0.0), mu(n), lz(n), ly((size_t)n * S, 0.0), vn1(n), keep((size_t)(K + 1) * n * S);
    const double inv = 1.0 / ((double)T * np);
    for (int seg = n_ck - 1; seg >= 0; --seg) {
        const int first = seg * K, last = std::min(T, first + K);
        std::copy(&ck[(size_t)seg * n * S], &ck[(size_t)(seg + 1) * n * S], y.begin());
        for (int i = 0; i < n; ++i) V[i] = y[(size_t)i * S];
        for (int s = first; s < last; ++s) {
            for (int i = 0; i < n; ++i) {
                y[(size_t)i * S] = V[i];
                std::copy(&y[(size_t)i * S], &y[(size_t)i * S] + S, &keep[((size_t)(s - first) * n + i) * S]);
            }
            if (!run_.step(s, y, V)) return -1;
        }
        for (int i = 0; i < n; ++i) keep[((size_t)(last - first) * n + i) * S] = V[i];
        for (int s = last - 1; s >= first; --s) {
            for (int i = 0; i < n; ++i) vn1[i] = keep[((size_t)(s + 1 - first) * n + i) * S];
            for (int k = 0; k < np; ++k)
                lam[probes[k]] += 2.0 * (vn1[probes[k]] - targets[(size_t)s * np + k]) * inv;
            std::fill(mu.begin(), mu.end(), 0.0);
            if (cg(run_.A, lam, mu, c.rtol, c.max_iterations, false) < 0) return -1;
            for (int e = 0; e < n - 1; ++e)
                grad[elem_region(e, n, R) * W + P] -=
                    (c.sigma / c.h) * (mu[e] - mu[e + 1]) * (vn1[e] - vn1[e + 1]);
            run_.Mm.mul(mu, lz);
            for (int i = 0; i < n; ++i) {
                const double* yn = &keep[((size_t)(s - first) * n + i) * S];
                const double* p = run_.params_of(i);
                double* gp = grad + node_region(i, n, R) * W;
                double* lyi = &ly[(size_t)i * S];
                const double st = run_.stim(i, s * c.dt) / c.am;
                double y1[S], dy[S];
                M::template rhs<double>(yn, st, c.cm, p, dy);
                for (int k = 0; k < S; ++k) y1[k] = k == 0 ? yn[0] : yn[k] + c.dt * dy[k];
                double lv = run_.ms * lz[i];
                const double lI = -c.am * lz[i];
                double gy[S] = {0.0};
                double gpp[P] = {0.0};
                M::template vjp_iionic<double>(y1, 0.0, c.cm, p, &lI, gy, gpp);
                lv += gy[0];
                for (int k = 1; k < S; ++k) lyi[k] += gy[k];
                double w[S], gf[S] = {0.0}, gpf[P] = {0.0};
                w[0] = 0.0;
                for (int k = 1; k < S; ++k) w[k] = lyi[k];
                M::template vjp_rhs<double>(yn, st, c.cm, p, w, gf, gpf);
                lv += c.dt * gf[0];
                for (int k = 1; k < S; ++k) lyi[k] += c.dt * gf[k];
                for (int k = 0; k < P; ++k) gp[k] += gpp[k] + c.dt * gpf[k];
                lam[i] = lv;
            }
        }
    }
    return 0;
}

// Directional derivative of the loss along dir (R x W) by a tangent-linear
// run: the ODE step and Iion on Dual numbers, then A dV' = M dz - dA V' for
// the new voltage's derivative (dA = dK along dir; CG to rtol from the last
// derivative).  The primal values follow the same arithmetic as run().
template <class M>
int tangent(const orc_cable_config& c, const double* prm, const double* dir, const int* probes, int np,
            const double* targets, double* dloss) {
    using Run = CableRun<M>;
    using chb::Dual;
    constexpr int S = Run::S, P = Run::P, W = Run::W;
    const int n = c.n_nodes, R = c.n_regions, T = c.n_steps;
    Run run_(c, prm);
    Tri dA;
    dA.d.assign(n, 0.0);
    dA.o.assign(n, 0.0);
    for (int e = 0; e < n - 1; ++e) {
        const double k = c.sigma * dir[elem_region(e, n, R) * W + P] / c.h;
        dA.d[e] += k;
        dA.d[e + 1] += k;
        dA.o[e] = -k;
    }
    std::vector<double> y((size_t)n * S), yd((size_t)n * S, 0.0), V(n), Vd(n, 0.0), z(n), zd(n), b(n), bd(n), t(n);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < S; ++k) y[(size_t)i * S + k] = M::kInitialStates[k];
    for (int i = 0; i < n; ++i) V[i] = y[(size_t)i * S];
    double acc = 0.0;
    for (int s = 0; s < T; ++s) {
        const double t0 = s * c.dt, t1 = t0 + c.dt;
        for (int i = 0; i < n; ++i) {
            const int r = node_region(i, n, R);
            Dual yy[S], pp[P], dy[S];
            for (int k = 0; k < S; ++k) yy[k] = Dual(y[(size_t)i * S + k], yd[(size_t)i * S + k]);
            yy[0] = Dual(V[i], Vd[i]);
            for (int k = 0; k < P; ++k) pp[k] = Dual(prm[r * W + k], dir[r * W + k]);
            M::template rhs<Dual>(yy, Dual(run_.stim(i, t0) / c.am), Dual(c.cm), pp, dy);
            for (int k = 1; k < S; ++k) yy[k] += Dual(c.dt) * dy[k];
            const Dual ii = M::template iionic<Dual>(yy, Dual(c.cm), pp);
            const Dual zz = Dual(run_.ms) * yy[0] + (Dual(-c.am) * ii - Dual(run_.stim(i, t1)));
            for (int k = 1; k < S; ++k) {
                y[(size_t)i * S + k] = yy[k].v;
                yd[(size_t)i * S + k] = yy[k].d;
            }
            z[i] = zz.v;
            zd[i] = zz.d;
        }
        run_.Mm.mul(z, b);
        if (cg(run_.A, b, V, c.rtol, c.max_iterations, true) < 0) return -1;
        run_.Mm.mul(zd, bd);
        dA.mul(V, t);
        for (int i = 0; i < n; ++i) bd[i] -= t[i];
        if (cg(run_.A, bd, Vd, c.rtol, c.max_iterations, true) < 0) return -1;
        for (int k = 0; k < np; ++k)
            acc += 2.0 * (V[probes[k]] - targets[(size_t)s * np + k]) * Vd[probes[k]];
    }
    *dloss = acc / ((double)T * np);
    return 0;
}

template <class M>
int tangent_gradient(const orc_cable_config& c, const double* prm, const int* probes, int np,
                     const double* targets, double* grad, int threads) {
    constexpr int W = M::kNumParams + 1;
    const int m = c.n_regions * W;
    std::vector<int> rc(m, 0);
    std::vector<std::thread> pool;
    const int nt = std::max(1, std::min(threads, m));
    for (int w = 0; w < nt; ++w) {
        pool.emplace_back([&, w]() {
            std::vector<double> dir(m);
            for (int k = w; k < m; k += nt) {
                std::fill(dir.begin(), dir.end(), 0.0);
                dir[k] = 1.0;
                rc[k] = tangent<M>(c, prm, dir.data(), probes, np, targets, &grad[k]);
            }
        });
    }
    for (auto& th : pool) th.join();
    for (int k = 0; k < m; ++k)
        if (rc[k]) return rc[k];
    return 0;
}

}  // namespace

extern "C" int orc_cable_tangent_gradient(const orc_cable_config* c, const double* params, const int* probes,
                                          int n_probes, const double* targets, double* grad, int threads) {
    if (!c || !params || !probes || n_probes < 1 || !targets || !grad || c->n_nodes < 2 || c->n_regions < 1 ||
        c->n_steps < 1)
        return -4;
    if (c->model == ORC_LR91)
        return tangent_gradient<chb::LuoRudy1991>(*c, params, probes, n_probes, targets, grad, threads);
    return tangent_gradient<chb::TenTusscher2006Epi>(*c, params, probes, n_probes, targets, grad, threads);
}

extern "C" int orc_cable_run(const orc_cable_config* c, const double* params, const int* probes, int n_probes,
                             const double* targets, double* loss, double* traces, double* grad) {
    if (!c || !params || (n_probes > 0 && !probes) || ((loss || grad) && !targets)) return -4;
    if (c->model == ORC_LR91)
        return run<chb::LuoRudy1991>(*c, params, probes, n_probes, targets, loss, traces, grad);
    return run<chb::TenTusscher2006Epi>(*c, params, probes, n_probes, targets, loss, traces, grad);
}
