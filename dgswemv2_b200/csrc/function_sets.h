// Problem function sets: initial condition ic_q(t,x,y), analytic source source_q(t,x,y),
// true solution true_q(t,x,y) and nodal bathymetry b(x,y).
//
// The reference swaps these in at compile time by copying headers over
// source/problem/SWE/problem_function_files/swe_{initial_condition,source,true_solution}_functions.hpp
// (examples/swe_manufactured_solution/build.sh:54-60). Here they are selected at run time by an
// integer id plus a small parameter block, and the same code runs on the host (setup, L2 projection
// of the initial condition) and on the device (function boundary condition, function source, L2 error).
//
// Bathymetry convention follows the reference: b is the still-water depth (positive below datum) and
// the total water column is h = ze + b (rkdg_swe_proc_volume.hpp:19-20).
#ifndef DGSW_FUNCTION_SETS_H
#define DGSW_FUNCTION_SETS_H

#include <math.h>

#if defined(__CUDACC__)
#define DGSW_HD __host__ __device__ __forceinline__
#else
#define DGSW_HD inline
#endif

#define DGSW_FN_PARAMS 16

enum dgsw_function_set_id {
    DGSW_FN_NONE = 0,                   // constant / default initial condition, no analytic source
    DGSW_FN_REFERENCE_MANUFACTURED = 1, // examples/swe_manufactured_solution/manufactured_swe_*.hpp
    DGSW_FN_MANUFACTURED_SINE = 2,      // ze = A sin(kx) cos(ky) cos(wt) on a square of side L
    DGSW_FN_THACKER_BOWL = 3,           // Thacker's oscillating paraboloid
    DGSW_FN_GAUSSIAN_HUMPS = 4,         // still water plus up to 3 Gaussian humps, q = 0
    DGSW_FN_COUNT = 5
};

struct dgsw_fn3 {
    double ze, qx, qy;
};

// ---------------------------------------------------------------------------------------------
// Set 1: the reference's own manufactured solution (g = 1, b = 2 on [-1,1]^2).
// Formulas restated from examples/swe_manufactured_solution/manufactured_swe_initial_condition_functions.hpp:34-36
// and manufactured_swe_source_functions.hpp:74-100.
// ---------------------------------------------------------------------------------------------
DGSW_HD dgsw_fn3 fn_refmms_true(double t, double x, double y) {
    dgsw_fn3 r;
    r.ze = exp(sin(3 * x) * sin(3 * y) - sin(3 * t));
    r.qx = cos(x - 4 * t);
    r.qy = sin(y + 4 * t);
    return r;
}

DGSW_HD dgsw_fn3 fn_refmms_source(double t, double x, double y) {
    const double E = exp(-sin(3 * t) + sin(3 * x) * sin(3 * y));
    const double H = 2 + E;
    dgsw_fn3 s;
    s.ze = -3 * E * cos(3 * t) + cos(4 * t + y) + sin(4 * t - x);
    s.qx = (cos(4 * t - x) * cos(4 * t + y)) / H - 4 * sin(4 * t - x) +
           (2 * cos(4 * t - x) * sin(4 * t - x)) / H + 3. * E * H * cos(3 * x) * sin(3 * y) -
           (3 * E * (cos(4 * t - x) * cos(4 * t - x)) * cos(3 * x) * sin(3 * y)) / (H * H) -
           (3 * E * cos(4 * t - x) * cos(3 * y) * sin(3 * x) * sin(4 * t + y)) / (H * H);
    s.qy = 4 * cos(4 * t + y) + 3. * E * H * cos(3 * y) * sin(3 * x) +
           (2 * cos(4 * t + y) * sin(4 * t + y)) / H + (sin(4 * t - x) * sin(4 * t + y)) / H -
           (3 * E * cos(4 * t - x) * cos(3 * x) * sin(3 * y) * sin(4 * t + y)) / (H * H) -
           (3 * E * cos(3 * y) * sin(3 * x) * (sin(4 * t + y) * sin(4 * t + y))) / (H * H);
    return s;
}

// ---------------------------------------------------------------------------------------------
// Set 2: manufactured standing wave on flat bathymetry H.
//   ze = A sin(kx) cos(ky) cos(wt),  qx = -B cos(kx) cos(ky) sin(wt),  qy = B sin(kx) sin(ky) sin(wt)
//   k = 2 pi / L, B = A w / (2k), so ze_t + div q = 0 exactly and the continuity source is zero.
// The momentum sources close the nonlinear equations:
//   S_x = qx_t + (qx^2/h)_x + (qx qy/h)_y + g h ze_x,   S_y = qy_t + (qx qy/h)_x + (qy^2/h)_y + g h ze_y
// params: [0]=L, [1]=A, [2]=H, [3]=w (0 -> k sqrt(2 g H)), [4]=g
// ---------------------------------------------------------------------------------------------
struct dgsw_sine_terms {
    double ze, zex, zey, zet, qx, qxx, qxy, qxt, qy, qyx, qyy, qyt;
};

DGSW_HD double fn_sine_omega(const double* P) {
    const double k = 2.0 * M_PI / P[0];
    return P[3] != 0.0 ? P[3] : k * sqrt(2.0 * P[4] * P[2]);
}

DGSW_HD dgsw_sine_terms fn_sine_terms(const double* P, double t, double x, double y) {
    const double k = 2.0 * M_PI / P[0];
    const double A = P[1];
    const double w = fn_sine_omega(P);
    const double B = A * w / (2.0 * k);
    const double sx = sin(k * x), cx = cos(k * x), sy = sin(k * y), cy = cos(k * y);
    const double st = sin(w * t), ct = cos(w * t);
    dgsw_sine_terms r;
    r.ze = A * sx * cy * ct;
    r.zex = A * k * cx * cy * ct;
    r.zey = -A * k * sx * sy * ct;
    r.zet = -A * w * sx * cy * st;
    r.qx = -B * cx * cy * st;
    r.qxx = B * k * sx * cy * st;
    r.qxy = B * k * cx * sy * st;
    r.qxt = -B * w * cx * cy * ct;
    r.qy = B * sx * sy * st;
    r.qyx = B * k * cx * sy * st;
    r.qyy = B * k * sx * cy * st;
    r.qyt = B * w * sx * sy * ct;
    return r;
}

DGSW_HD dgsw_fn3 fn_sine_true(const double* P, double t, double x, double y) {
    dgsw_sine_terms s = fn_sine_terms(P, t, x, y);
    dgsw_fn3 r;
    r.ze = s.ze;
    r.qx = s.qx;
    r.qy = s.qy;
    return r;
}

DGSW_HD dgsw_fn3 fn_sine_source(const double* P, double t, double x, double y) {
    dgsw_sine_terms s = fn_sine_terms(P, t, x, y);
    const double g = P[4];
    const double h = s.ze + P[2];
    const double ih = 1.0 / h;
    const double ih2 = ih * ih;
    dgsw_fn3 r;
    r.ze = s.zet + s.qxx + s.qyy;  // identically zero up to rounding
    r.qx = s.qxt + (2.0 * s.qx * s.qxx * ih - s.qx * s.qx * s.zex * ih2) +
           ((s.qxy * s.qy + s.qx * s.qyy) * ih - s.qx * s.qy * s.zey * ih2) + g * h * s.zex;
    r.qy = s.qyt + ((s.qxx * s.qy + s.qx * s.qyx) * ih - s.qx * s.qy * s.zex * ih2) +
           (2.0 * s.qy * s.qyy * ih - s.qy * s.qy * s.zey * ih2) + g * h * s.zey;
    return r;
}

// ---------------------------------------------------------------------------------------------
// Set 3: Thacker (1981) oscillating paraboloid in a bowl of depth b(r) = h0 (1 - r^2/a^2).
//   A = ((h0+eta0)^2 - h0^2) / ((h0+eta0)^2 + h0^2),  w = sqrt(8 g h0) / a
//   ze(r,t) = h0 [ sqrt(1-A^2)/(1-A cos wt) - 1 - r^2/a^2 ((1-A^2)/(1-A cos wt)^2 - 1) ]
//   u = x w A sin(wt) / (2 (1 - A cos wt)),  v = y (same factor)
// Where the analytic column ze + b is not positive the cell is dry: ze = -b, q = 0.
// params: [0]=h0, [1]=a, [2]=eta0, [3]=g, [4]=xc, [5]=yc
// ---------------------------------------------------------------------------------------------
DGSW_HD double fn_thacker_bath(const double* P, double x, double y) {
    const double dx = x - P[4], dy = y - P[5];
    const double r2 = dx * dx + dy * dy;
    return P[0] * (1.0 - r2 / (P[1] * P[1]));
}

DGSW_HD double fn_thacker_omega(const double* P) { return sqrt(8.0 * P[3] * P[0]) / P[1]; }

DGSW_HD dgsw_fn3 fn_thacker_true(const double* P, double t, double x, double y) {
    const double h0 = P[0], a = P[1], eta0 = P[2];
    const double hp = (h0 + eta0) * (h0 + eta0);
    const double A = (hp - h0 * h0) / (hp + h0 * h0);
    const double w = fn_thacker_omega(P);
    const double dx = x - P[4], dy = y - P[5];
    const double r2 = dx * dx + dy * dy;
    const double den = 1.0 - A * cos(w * t);
    double ze = h0 * (sqrt(1.0 - A * A) / den - 1.0 - r2 / (a * a) * ((1.0 - A * A) / (den * den) - 1.0));
    const double b = fn_thacker_bath(P, x, y);
    dgsw_fn3 r;
    if (ze + b > 0.0) {
        const double fac = w * A * sin(w * t) / (2.0 * den);
        r.ze = ze;
        r.qx = (ze + b) * dx * fac;
        r.qy = (ze + b) * dy * fac;
    } else {
        r.ze = -b;
        r.qx = 0.0;
        r.qy = 0.0;
    }
    return r;
}

// ---------------------------------------------------------------------------------------------
// Set 4: still water ze0 plus up to three Gaussian humps, zero momentum.
// params: [0]=ze0, then per hump i<3: [1+4i]=amplitude, [2+4i]=xc, [3+4i]=yc, [4+4i]=width
// A hump with zero width is ignored.
// ---------------------------------------------------------------------------------------------
DGSW_HD dgsw_fn3 fn_humps_true(const double* P, double x, double y) {
    double ze = P[0];
    for (int i = 0; i < 3; ++i) {
        const double w = P[4 + 4 * i];
        if (w > 0.0) {
            const double dx = x - P[2 + 4 * i], dy = y - P[3 + 4 * i];
            ze += P[1 + 4 * i] * exp(-(dx * dx + dy * dy) / (2.0 * w * w));
        }
    }
    dgsw_fn3 r;
    r.ze = ze;
    r.qx = 0.0;
    r.qy = 0.0;
    return r;
}

// ---------------------------------------------------------------------------------------------
// Dispatch. ic_q is also the exterior state of the function boundary condition
// (rkdg_swe_bc_function.hpp:33-50 evaluates SWE::ic_q(t, pt) at the edge Gauss points).
// ---------------------------------------------------------------------------------------------
DGSW_HD dgsw_fn3 dgsw_fn_true(int id, const double* P, double t, double x, double y) {
    switch (id) {
        case DGSW_FN_REFERENCE_MANUFACTURED:
            return fn_refmms_true(t, x, y);
        case DGSW_FN_MANUFACTURED_SINE:
            return fn_sine_true(P, t, x, y);
        case DGSW_FN_THACKER_BOWL:
            return fn_thacker_true(P, t, x, y);
        case DGSW_FN_GAUSSIAN_HUMPS:
            return fn_humps_true(P, x, y);
        default: {
            dgsw_fn3 r;
            r.ze = 0.0;
            r.qx = 0.0;
            r.qy = 0.0;
            return r;
        }
    }
}

DGSW_HD dgsw_fn3 dgsw_fn_ic(int id, const double* P, double t, double x, double y) { return dgsw_fn_true(id, P, t, x, y); }

DGSW_HD dgsw_fn3 dgsw_fn_source(int id, const double* P, double t, double x, double y) {
    switch (id) {
        case DGSW_FN_REFERENCE_MANUFACTURED:
            return fn_refmms_source(t, x, y);
        case DGSW_FN_MANUFACTURED_SINE:
            return fn_sine_source(P, t, x, y);
        default: {
            dgsw_fn3 r;
            r.ze = 0.0;
            r.qx = 0.0;
            r.qy = 0.0;
            return r;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Split evaluation for the device: the time-only factors of a set are computed once per stage
// (dgsw_fn_prepare), the space-dependent part per point in the kernel's precision (dgsw_fn_eval).
// Same formulas as above; only the time factors are hoisted out of the point loop.
// ---------------------------------------------------------------------------------------------
struct dgsw_fn_time {
    double t;
    double s[6];
};

DGSW_HD dgsw_fn_time dgsw_fn_prepare(int id, const double* P, double t) {
    dgsw_fn_time T;
    T.t = t;
    for (int i = 0; i < 6; ++i) T.s[i] = 0.0;
    if (id == DGSW_FN_MANUFACTURED_SINE) {
        const double w = fn_sine_omega(P);
        T.s[0] = sin(w * t);
        T.s[1] = cos(w * t);
        T.s[2] = w;
    } else if (id == DGSW_FN_THACKER_BOWL) {
        const double h0 = P[0], eta0 = P[2];
        const double hp = (h0 + eta0) * (h0 + eta0);
        const double A = (hp - h0 * h0) / (hp + h0 * h0);
        const double w = fn_thacker_omega(P);
        T.s[0] = 1.0 - A * cos(w * t);  // den
        T.s[1] = sin(w * t);
        T.s[2] = A;
        T.s[3] = w;
    }
    return T;
}

DGSW_HD void dgsw_sincos(double a, double* s, double* c) {
#if defined(__CUDA_ARCH__)
    sincos(a, s, c);
#else
    *s = sin(a);
    *c = cos(a);
#endif
}
DGSW_HD void dgsw_sincos(float a, float* s, float* c) {
#if defined(__CUDA_ARCH__) && defined(DGSW_ACCURATE_SINCOS)
    sincosf(a, s, c);
#elif defined(__CUDA_ARCH__)
    // FP32 bulk path: reduce to [-pi, pi] with a two-term Cody-Waite split of 2 pi (6.28125 is exact in
    // FP32 with a short mantissa, so n * 6.28125 is exact for the small n met here), then the hardware
    // sine/cosine, whose absolute error there is a few 1e-7 - below the FP32 state's own rounding
    const float n = rintf(a * 0.15915494309189535f);
    float r = fmaf(-n, 6.28125f, a);
    r = fmaf(-n, 1.9353071795864769e-3f, r);
    __sincosf(r, s, c);
#else
    *s = sinf(a);
    *c = cosf(a);
#endif
}

// source = 0: ic_q / true_q;  source = 1: source_q.  R = double or float.
template <typename R>
DGSW_HD void dgsw_fn_eval(int id, const double* P, const dgsw_fn_time& T, int source, R x, R y, R out[3]) {
    out[0] = out[1] = out[2] = R(0);
    if (id == DGSW_FN_MANUFACTURED_SINE) {
        const R k = (R)(2.0 * M_PI / P[0]);
        const R A = (R)P[1], w = (R)T.s[2];
        const R B = (R)(P[1] * T.s[2] / (2.0 * (2.0 * M_PI / P[0])));
        const R st = (R)T.s[0], ct = (R)T.s[1];
        R sx, cx, sy, cy;
        dgsw_sincos(k * x, &sx, &cx);
        dgsw_sincos(k * y, &sy, &cy);
        const R ze = A * sx * cy * ct;
        const R qx = -B * cx * cy * st;
        const R qy = B * sx * sy * st;
        if (!source) {
            out[0] = ze;
            out[1] = qx;
            out[2] = qy;
            return;
        }
        const R zex = A * k * cx * cy * ct, zey = -A * k * sx * sy * ct, zet = -A * w * sx * cy * st;
        const R qxx = B * k * sx * cy * st, qxy = B * k * cx * sy * st, qxt = -B * w * cx * cy * ct;
        const R qyx = B * k * cx * sy * st, qyy = B * k * sx * cy * st, qyt = B * w * sx * sy * ct;
        const R g = (R)P[4];
        const R h = ze + (R)P[2];
        const R ih = R(1) / h;
        const R ih2 = ih * ih;
        out[0] = zet + qxx + qyy;
        out[1] = qxt + (R(2) * qx * qxx * ih - qx * qx * zex * ih2) + ((qxy * qy + qx * qyy) * ih - qx * qy * zey * ih2) +
                 g * h * zex;
        out[2] = qyt + ((qxx * qy + qx * qyx) * ih - qx * qy * zex * ih2) + (R(2) * qy * qyy * ih - qy * qy * zey * ih2) +
                 g * h * zey;
        return;
    }
    if (id == DGSW_FN_THACKER_BOWL) {
        if (source) return;
        const R h0 = (R)P[0], a = (R)P[1];
        const R dx = x - (R)P[4], dy = y - (R)P[5];
        const R r2 = dx * dx + dy * dy;
        const R den = (R)T.s[0], A = (R)T.s[2];
        const R ze = h0 * ((R)sqrt(1.0 - T.s[2] * T.s[2]) / den - R(1) - r2 / (a * a) * ((R(1) - A * A) / (den * den) - R(1)));
        const R b = h0 * (R(1) - r2 / (a * a));
        if (ze + b > R(0)) {
            const R fac = (R)T.s[3] * A * (R)T.s[1] / (R(2) * den);
            out[0] = ze;
            out[1] = (ze + b) * dx * fac;
            out[2] = (ze + b) * dy * fac;
        } else {
            out[0] = -b;
        }
        return;
    }
    if (id == DGSW_FN_GAUSSIAN_HUMPS) {
        if (source) return;
        R ze = (R)P[0];
        for (int i = 0; i < 3; ++i) {
            const R wd = (R)P[4 + 4 * i];
            if (wd > R(0)) {
                const R dx = x - (R)P[2 + 4 * i], dy = y - (R)P[3 + 4 * i];
                ze += (R)P[1 + 4 * i] * (R)exp((double)(-(dx * dx + dy * dy) / (R(2) * wd * wd)));
            }
        }
        out[0] = ze;
        return;
    }
    if (id == DGSW_FN_REFERENCE_MANUFACTURED) {
        const dgsw_fn3 f = source ? fn_refmms_source(T.t, (double)x, (double)y) : fn_refmms_true(T.t, (double)x, (double)y);
        out[0] = (R)f.ze;
        out[1] = (R)f.qx;
        out[2] = (R)f.qy;
    }
}


#endif
