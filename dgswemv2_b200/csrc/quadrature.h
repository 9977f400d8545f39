// Quadrature rules on the master triangle (-1,-1),(1,-1),(-1,1) and on [-1,1]. Host-side C++.
//
// * Dunavant symmetric rules of degree 1..5 (the degrees RKDG p = 1, 2 use are 2p = 2 and 4).
//   The point/weight data are Dunavant's published 15-digit values; the reference carries the same
//   data in source/integration/integrations_2D/integration_dunavant_2D.cpp:354-392 and maps them to
//   the master triangle by z = 2*bary - 1, w = 2*w_bary with the 1/3/6-orbit expansion of :4-76.
//   The values have to be the same for results to agree, so they are restated as data here.
// * Gauss-Legendre rules with n points, computed by Newton iteration on P_n in long double
//   (the reference tabulates them, integration_gausslegendre_1D.cpp:32-; the reference picks
//   n = ceil((degree+1)/2), :28-30).
// * A collapsed (conical) product rule of any degree, Gauss-Legendre in one direction and
//   Gauss-Jacobi(1,0) in the other, used where the reference asks for a Dunavant rule of degree
//   above 5 (the degree-20 rule of Element::ComputeResidualL2, element.hpp:551). Both rules are
//   exact to the same polynomial degree.
#ifndef DGSW_QUADRATURE_H
#define DGSW_QUADRATURE_H

#include <cmath>
#include <stdexcept>
#include <vector>

namespace dgsw {

struct Rule2D {
    std::vector<double> w;   // weights (sum = 2, the master triangle area)
    std::vector<double> z1;  // master coordinates
    std::vector<double> z2;
};

struct Rule1D {
    std::vector<double> w;  // weights on [-1,1]
    std::vector<double> z;
};

// Jacobi polynomial P_n^{(a,0)}(x) and P_{n-1}^{(a,0)}(x) by the three-term recurrence
inline void jacobi_a0(int n, long double a, long double x, long double& pn, long double& pm) {
    long double p0 = 1.0L, p1 = 0.5L * (a + (a + 2) * x);
    if (n == 0) {
        pn = 1.0L;
        pm = 0.0L;
        return;
    }
    for (int k = 1; k < n; ++k) {
        long double a1 = 2 * (k + 1) * (k + a + 1) * (2 * k + a);
        long double a2 = (2 * k + a + 1) * (a * a);
        long double a3 = (2 * k + a) * (2 * k + a + 1) * (2 * k + a + 2);
        long double a4 = 2 * (k + a) * k * (2 * k + a + 2);
        long double pk1 = ((a2 + a3 * x) * p1 - a4 * p0) / a1;
        p0 = p1;
        p1 = pk1;
    }
    pn = p1;
    pm = p0;
}

// Gauss-Jacobi nodes/weights for the weight (1-x)^a on [-1,1] (a = 0: Gauss-Legendre), computed by
// Newton iteration with deflation against the roots already found, in long double.
inline void gauss_jacobi(int n, int alpha, std::vector<long double>& x, std::vector<long double>& w) {
    x.assign(n, 0.0L);
    w.assign(n, 0.0L);
    const long double pi = 3.141592653589793238462643383279502884L;
    const long double a = alpha;
    for (int i = 0; i < n; ++i) {
        long double r = -std::cos(pi * (i + 0.75L) / (n + 0.5L));
        for (int it = 0; it < 500; ++it) {
            long double pn, pm;
            jacobi_a0(n, a, r, pn, pm);
            long double dp = (n * (a - (2 * n + a) * r) * pn + 2 * (n + a) * n * pm) / ((2 * n + a) * (1 - r * r));
            long double defl = 0.0L;
            for (int j = 0; j < i; ++j) defl += 1.0L / (r - x[j]);
            long double dr = pn / (dp - pn * defl);
            r -= dr;
            if (std::fabs(dr) < 1e-32L) break;
        }
        x[i] = r;
        long double pn, pm;
        jacobi_a0(n, a, r, pn, pm);
        long double dp = (n * (a - (2 * n + a) * r) * pn + 2 * (n + a) * n * pm) / ((2 * n + a) * (1 - r * r));
        // weight for (1-x)^a, b = 0:  w = 2^{a+1} / ((1 - x^2) P_n'(x)^2)
        w[i] = std::pow(2.0L, a + 1) / ((1 - r * r) * dp * dp);
    }
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j)
            if (x[j] < x[i]) {
                std::swap(x[i], x[j]);
                std::swap(w[i], w[j]);
            }
}

inline Rule1D gauss_legendre(int npt) {
    std::vector<long double> x, w;
    gauss_jacobi(npt, 0, x, w);
    Rule1D r;
    for (int i = 0; i < npt; ++i) {
        // symmetrise so that z[n-1-i] == -z[i] exactly, as in the tabulated rules
        long double xs = 0.5L * (x[i] - x[npt - 1 - i]);
        long double ws = 0.5L * (w[i] + w[npt - 1 - i]);
        r.z.push_back((double)xs);
        r.w.push_back((double)ws);
    }
    if (npt % 2 == 1) r.z[npt / 2] = 0.0;
    return r;
}

// number of GL points used for a requested polynomial degree (integration_gausslegendre_1D.cpp:28-30)
inline int gauss_legendre_npt(int degree) { return (int)std::ceil(((double)degree + 1) / 2); }

inline Rule1D gauss_legendre_degree(int degree) { return gauss_legendre(gauss_legendre_npt(degree)); }

// collapsed product rule of the given polynomial degree on the master triangle
inline Rule2D conical_rule(int degree) {
    int n = degree / 2 + 1;
    std::vector<long double> xa, wa, xb, wb;
    gauss_jacobi(n, 0, xa, wa);  // eta1 direction
    gauss_jacobi(n, 1, xb, wb);  // eta2 direction, weight (1 - eta2)
    Rule2D r;
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i) {
            long double e1 = xa[i], e2 = xb[j];
            long double z1 = 0.5L * (1 + e1) * (1 - e2) - 1;
            long double z2 = e2;
            r.z1.push_back((double)z1);
            r.z2.push_back((double)z2);
            r.w.push_back((double)(0.5L * wa[i] * wb[j]));
        }
    }
    return r;
}

// Dunavant barycentric orbit data: multiplicity (1, 3 or 6), weight, barycentric (a, b, c)
struct DunavantOrbit {
    int mult;
    double w;
    double a, b, c;
};

inline std::vector<DunavantOrbit> dunavant_orbits(int degree) {
    std::vector<DunavantOrbit> o;
    if (degree == 0 || degree == 1) {
        o.push_back({1, 1.000000000000000, 0.333333333333333, 0.333333333333333, 0.333333333333333});
    } else if (degree == 2) {
        o.push_back({3, 0.333333333333333, 0.666666666666667, 0.166666666666667, 0.166666666666667});
    } else if (degree == 3) {
        o.push_back({1, -0.562500000000000, 0.333333333333333, 0.333333333333333, 0.333333333333333});
        o.push_back({3, 0.520833333333333, 0.600000000000000, 0.200000000000000, 0.200000000000000});
    } else if (degree == 4) {
        o.push_back({3, 0.223381589678011, 0.108103018168070, 0.445948490915965, 0.445948490915965});
        o.push_back({3, 0.109951743655322, 0.816847572980459, 0.091576213509771, 0.091576213509771});
    } else if (degree == 5) {
        o.push_back({1, 0.225000000000000, 0.333333333333333, 0.333333333333333, 0.333333333333333});
        o.push_back({3, 0.132394152788506, 0.059715871789770, 0.470142064105115, 0.470142064105115});
        o.push_back({3, 0.125939180544827, 0.797426985353087, 0.101286507323456, 0.101286507323456});
    }
    return o;
}

inline bool dunavant_has_degree(int degree) { return degree >= 0 && degree <= 5; }

// Dunavant rule of the given degree mapped to the master triangle; falls back to the conical rule
// of the same degree above 5.
inline Rule2D triangle_rule(int degree) {
    if (!dunavant_has_degree(degree)) return conical_rule(degree);
    Rule2D r;
    for (const DunavantOrbit& ob : dunavant_orbits(degree)) {
        const double w = 2 * ob.w;
        auto push = [&](double p, double q) {
            r.w.push_back(w);
            r.z1.push_back(2 * p - 1);
            r.z2.push_back(2 * q - 1);
        };
        if (ob.mult == 1) {
            push(ob.a, ob.b);
        } else if (ob.mult == 3) {
            push(ob.a, ob.b);
            push(ob.b, ob.c);
            push(ob.c, ob.a);
        } else {
            push(ob.a, ob.b);
            push(ob.b, ob.c);
            push(ob.c, ob.a);
            push(ob.b, ob.a);
            push(ob.c, ob.b);
            push(ob.a, ob.c);
        }
    }
    return r;
}

}  // namespace dgsw

#endif
