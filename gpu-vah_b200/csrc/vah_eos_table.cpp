// vah_eos_table.cpp -- host builder of the tabulated crossover equation of state.
//
// The reference ships only closed-form EoS fits (rhic/src/EquationOfState.cpp:
// 31-201); the 3+1D workloads use a tabulated crossover instead, defined here:
//
//   c_s^2(T) = 1/3 - D / (1 + (T/Tc)^4),   D = 1/3 - 0.15,  Tc = 155 MeV
//
// i.e. a hadron-gas-like c_s^2 = 0.15 well below Tc and the conformal 1/3 well
// above it. With d ln s / d ln T = 1/c_s^2 the entropy density is closed-form,
//
//   s(T) = s_inf tau^3 (tau^4 / (tau^4 + a))^(9D/(4a)),  tau = T/Tc, a = 1 - 3D,
//
// normalised to the reference's conformal gas at high T
// (s -> (4/3) 13.8997 T^3, EquationOfState.h:16). The pressure
// p(T) = int_0^T s dT' is integrated numerically and e = T s - p.
//
// Layout (include/vah.h): tab[0] = n, tab[1] = ln e_0, tab[2] = 1/d(ln e),
// tab[3] = d(ln e), tab[4] = e_0, tab[5] = ln e_{n-1}, tab[6] = e_{n-1},
// tab[7] = 0, then p[n], T[n], c_s^2[n] on nodes uniform in ln e from
// T = 5 MeV to T = 5 GeV. Units: T in fm^-1, e and p in fm^-4.
#include <cmath>
#include <vector>

#include "vah.h"

namespace {

constexpr double kHbarc = 0.197326938;
constexpr double kEosFactor = 13.8997;
constexpr double kDelta = 1.0 / 3.0 - 0.15;
constexpr double kA = 1.0 - 3.0 * kDelta;
const double kExpo = 9.0 * kDelta / (4.0 * kA);
const double kTc = 0.155 / kHbarc;
const double kSinf = 4.0 / 3.0 * kEosFactor * kTc * kTc * kTc;

double cs2_of(double T) {
    double tau = T / kTc;
    double t4 = tau * tau * tau * tau;
    return 1.0 / 3.0 - kDelta / (1.0 + t4);
}

double s_of(double T) {
    double tau = T / kTc;
    double t4 = tau * tau * tau * tau;
    return kSinf * tau * tau * tau * std::pow(t4 / (t4 + kA), kExpo);
}

// int_{T0}^{T1} s dT by Simpson on ln T over one short interval.
double simpson_piece(double T0, double T1) {
    double l0 = std::log(T0), l1 = std::log(T1), lm = 0.5 * (l0 + l1);
    double Tm = std::exp(lm);
    return (l1 - l0) / 6.0 * (s_of(T0) * T0 + 4.0 * s_of(Tm) * Tm + s_of(T1) * T1);
}

}  // namespace

extern "C" int vah_eos_table_build(int n, double *out, size_t out_len) {
    if (n < 16 || out == nullptr || out_len < VAH_EOS_TABLE_LEN(n)) return VAH_ERR_ARG;

    // Fine ln T grid from 1 MeV to 10 GeV; p starts from the c_s^2 = 0.15
    // power law p = 3 T s / 23 (s ~ T^(20/3)) at the lower end.
    const int M = 1 << 17;
    const double lt0 = std::log(0.001 / kHbarc), lt1 = std::log(10.0 / kHbarc);
    const double h = (lt1 - lt0) / M;
    std::vector<double> Tf(M + 1), pf(M + 1), ef(M + 1);
    for (int k = 0; k <= M; ++k) Tf[k] = std::exp(lt0 + h * k);
    pf[0] = 3.0 * Tf[0] * s_of(Tf[0]) / 23.0;
    for (int k = 0; k < M; ++k) pf[k + 1] = pf[k] + simpson_piece(Tf[k], Tf[k + 1]);
    for (int k = 0; k <= M; ++k) ef[k] = Tf[k] * s_of(Tf[k]) - pf[k];

    auto e_at = [&](int k, double T, double *p_out) {
        double p = pf[k] + simpson_piece(Tf[k], T);
        *p_out = p;
        return T * s_of(T) - p;
    };
    // e(T) on the fine grid, refined inside a grid interval by Newton steps.
    auto solve_T = [&](double e_target, double *p_out) {
        int lo = 0, hi = M;
        while (hi - lo > 1) {
            int mid = (lo + hi) / 2;
            if (ef[mid] <= e_target) lo = mid; else hi = mid;
        }
        double w = (std::log(e_target) - std::log(ef[lo])) / (std::log(ef[lo + 1]) - std::log(ef[lo]));
        double T = std::exp(std::log(Tf[lo]) + w * h);
        double p = 0.0;
        for (int it = 0; it < 4; ++it) {
            double e = e_at(lo, T, &p);
            double dedT = s_of(T) / cs2_of(T);
            T -= (e - e_target) / dedT;
        }
        e_at(lo, T, &p);
        *p_out = p;
        return T;
    };

    const double Tlo = 0.005 / kHbarc, Thi = 5.0 / kHbarc;
    double plo, phi;
    // e at the two end temperatures (bracketing interval found by search)
    auto e_of_T = [&](double T, double *p_out) {
        int k = (int)std::floor((std::log(T) - lt0) / h);
        if (k < 0) k = 0;
        if (k >= M) k = M - 1;
        return e_at(k, T, p_out);
    };
    const double lne0 = std::log(e_of_T(Tlo, &plo));
    const double lne1 = std::log(e_of_T(Thi, &phi));
    const double dl = (lne1 - lne0) / (n - 1);

    double *P = out + VAH_EOS_TABLE_HEADER, *T = P + n, *C = T + n;
    for (int i = 0; i < n; ++i) {
        double et = std::exp(lne0 + dl * i);
        double p;
        double Ti = solve_T(et, &p);
        P[i] = p;
        T[i] = Ti;
        C[i] = cs2_of(Ti);
    }
    out[0] = (double)n;
    out[1] = lne0;
    out[2] = 1.0 / dl;
    out[3] = dl;
    out[4] = std::exp(lne0);
    out[5] = lne0 + dl * (n - 1);
    out[6] = std::exp(out[5]);
    out[7] = 0.0;
    return VAH_OK;
}
