// zolotarev.cpp -- Zolotarev optimal rational approximation of Y^-1/2 on
// [r_a^2, r_b^2] (M. Luscher, "Computational strategies in lattice QCD",
// hep-lat/0406022, sect. 3), the coefficients of get_rhmc_params
// (src/QED2dRHMC.jl:1-121).  The reference evaluates K(m), sn(u|m), cn(u|m)
// with Elliptic.jl 1.0.1; here they come from the arithmetic-geometric mean:
// K(m) = pi / (2 AGM(1, sqrt(1-m))), and sn, cn by the descending Landen
// scheme (Abramowitz & Stegun 16.4).  Host code, FP64.
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"

namespace qed2d {
namespace {

struct Elliptic {
    double m;
    std::vector<double> a, c;   // AGM sequence for sn/cn
    double K;
    explicit Elliptic(double m_) : m(m_) {
        double aa = 1.0, bb = std::sqrt(1.0 - m), cc = std::sqrt(m);
        a.push_back(aa);
        c.push_back(cc);
        while (std::fabs(cc) > 1e-17 * aa && a.size() < 63) {
            const double an = 0.5 * (aa + bb), bn = std::sqrt(aa * bb);
            cc = 0.5 * (aa - bb);
            aa = an;
            bb = bn;
            a.push_back(aa);
            c.push_back(cc);
        }
        K = M_PI / (2.0 * aa);
    }
    void sncn(double u, double& sn, double& cn) const {
        const int N = (int)a.size() - 1;
        double phi = std::ldexp(a[N] * u, N);
        for (int k = N; k >= 1; k--) phi = 0.5 * (phi + std::asin(c[k] / a[k] * std::sin(phi)));
        sn = std::sin(phi);
        cn = std::cos(phi);
    }
};

}  // namespace

int zolotarev_params(int n, double r_a, double r_b, qed2d_rhmc_params* out) {
    if (!out || n < 1 || n > QED2D_MAXPOLES || !(r_a > 0.0) || !(r_b > r_a)) return QED2D_ERR_BAD_ARG;
    std::memset(out, 0, sizeof(*out));
    const double eps = (r_a / r_b) * (r_a / r_b);
    const double k = std::sqrt(1.0 - eps);            // k(eps)        :2
    const Elliptic E(k * k);
    const double v = E.K / (2.0 * n + 1.0);           // v(n, eps)     :3
    std::vector<double> sn2(2 * n + 2), cn2(2 * n + 2);
    for (int r = 1; r <= 2 * n + 1; r++) {
        double s, c;
        E.sncn(r * v, s, c);
        sn2[r] = s * s;
        cn2[r] = c * c;
    }
    auto a_r = [&](int r) { return cn2[r] / sn2[r]; };   // :4
    auto c_r = [&](int r) { return sn2[r]; };           // :5
    std::vector<double> mu(n + 1), nu(n + 1);
    for (int j = 1; j <= n; j++) {
        mu[j] = r_b * std::sqrt(a_r(2 * j));            // :8
        nu[j] = r_b * std::sqrt(a_r(2 * j - 1));        // :9
    }
    double d = std::pow(k, 2 * n + 1);                  // d(n, eps)     :60-68
    for (int i = 1; i <= 2 * n + 1; i += 2) d *= c_r(i) * c_r(i);
    const double den = 1.0 + std::sqrt(1.0 - d * d);
    double A = 2.0 / den;                               // A(n, eps)     :72-84
    for (int i = 1; i <= 2 * n - 1; i += 2) A *= c_r(i);
    for (int i = 2; i <= 2 * n; i += 2) A *= 1.0 / c_r(i);
    out->r_b = r_b;
    out->n = n;
    out->eps = eps;
    out->A = A;
    out->delta = d * d / (den * den);                   // delta(n, eps) :70
    for (int j = 1; j <= n; j++) {
        double res = nu[j] * nu[j] - mu[j] * mu[j];     // rho_mu        :11-25
        for (int m = 1; m <= n; m++)
            if (m != j) res *= (nu[m] * nu[m] - mu[j] * mu[j]) / (mu[m] * mu[m] - mu[j] * mu[j]);
        out->mu[j - 1] = mu[j];
        out->nu[j - 1] = nu[j];
        out->rho[j - 1] = res;
    }
    out->reweighting_N = 1;        // defaults of get_rhmc_params, :93
    out->reweighting_Taylor = 5;
    return QED2D_OK;
}

}  // namespace qed2d

// Elliptic.K(m) and Jacobi.sn/cn(u, m) of Elliptic.jl, the functions behind the
// reference's Zolotarev helpers (src/QED2dRHMC.jl:3-5), on the same AGM/Landen
// restatement as the coefficients above.
extern "C" int qed2d_ellip_K(double m, double* K) {
    if (!K || !(m >= 0.0 && m < 1.0)) {
        qed2d::set_error("ellip_K: need 0 <= m < 1 and a non-NULL output");
        return QED2D_ERR_BAD_ARG;
    }
    *K = qed2d::Elliptic(m).K;
    return QED2D_OK;
}

extern "C" int qed2d_ellip_sncn(double u, double m, double* sn, double* cn) {
    if (!sn || !cn || !(m >= 0.0 && m < 1.0) || !std::isfinite(u)) {
        qed2d::set_error("ellip_sncn: need 0 <= m < 1, finite u and non-NULL outputs");
        return QED2D_ERR_BAD_ARG;
    }
    qed2d::Elliptic(m).sncn(u, *sn, *cn);
    return QED2D_OK;
}
