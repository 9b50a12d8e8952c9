// The reference's equation registry as device code.
//
// The reference's operator interface is a compile-time "Eq concept" resolved
// in wos_sample (include/wos/wos.hpp:54-138): has_source / has_screening
// flags, boundary(p[, boundary_id]), source(p), green(sphere, x, y),
// green_mass(R), sample_green(sphere, rng), screening_factor(R) and, in 2D,
// source_may_intersect(sphere).  Each struct below is one registry entry for
// one dimension with exactly those members (src/equations/laplace.cpp:12-43,
// poisson.cpp:15-118, screened_poisson.cpp:40-141, helmholtz.cpp:15-78);
// Green kernels follow include/wos/poisson.hpp:12-51 and
// include/wos/screened.hpp:14-156.
//
// Member functions are templates on the arithmetic type T: the exact path
// instantiates them with double (expression shapes follow the reference so
// they round identically), the fast path with float.  Random draws come from
// an Rng with unit() in [0, 1) and unit_open() in (0, 1).
#pragma once
#include "special.cuh"

namespace wosb {

enum : int {
    kLaplace = 0,
    kPoisson = 1,
    kScreened = 2,
    kHelmholtz = 3,
    kTransient = 4,
    kPlate = 5
};
enum : int { kUniform = 0, kGreen = 1, kMis = 2 };

template <typename T>
struct V3 {
    T x, y, z;
};

template <typename T>
__device__ __forceinline__ T harmonic_y5(T x, T y, T z) {
    // src/equations/laplace.cpp:30-36
    const T r_sq = x * x + y * y;
    const T y50 = z * (T(8) * z * z * z * z - T(40) * z * z * r_sq + T(15) * r_sq * r_sq);
    const T y5m3 = (T(8) * z * z - r_sq) * y * (T(3) * x * x - y * y);
    return y50 + T(4) * y5m3;
}

template <int DIM, typename T>
__device__ __forceinline__ T dist(V3<T> a, V3<T> b) {
    if (DIM == 2) return sqrt((a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y));
    return sqrt((a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y) + (a.z - b.z) * (a.z - b.z));
}

// Angles: the exact path forms theta in double and calls cos/sin like the
// reference.  FAST_FP64 uses sincospi on 2u.  FAST_FP32 takes the hardware
// sine/cosine of 2 pi u - pi, an angle in [-pi, pi] where their absolute error
// is documented as at most 2^-21.41 (a uniform angle turned by pi is still
// uniform).  That moves a step point by under 4e-7 R, far inside the
// 2^-10 relative margin of every FP32 radius; inside the epsilon shell the
// walk re-projects in FP64 anyway.
template <typename T>
__device__ __forceinline__ void sincos_2pi(T u, T &s, T &c);
template <>
__device__ __forceinline__ void sincos_2pi<float>(float u, float &s, float &c) {
    __sincosf(fmaf(u, 6.28318531f, -3.14159265f), &s, &c);
}
template <>
__device__ __forceinline__ void sincos_2pi<double>(double u, double &s, double &c) {
    sincospi(2.0 * u, &s, &c);
}

// ---------------------------------------------------------------- sampling

// Exit point on the sphere, src/wos.cpp:9-30.
template <int DIM, bool EXACT, typename T, class Rng>
__device__ __forceinline__ V3<T> sphere_step(V3<T> c, T R, Rng &rng) {
    if (DIM == 2) {
        if constexpr (EXACT) {
            const double theta = rng.unit() * 2 * kPi;
            return V3<T>{c.x + R * cos(theta), c.y + R * sin(theta), T(0)};
        }
        T s, co;
        sincos_2pi<T>(rng.unit(), s, co);
        return V3<T>{c.x + R * co, c.y + R * s, T(0)};
    } else {
        const T u = rng.unit();
        const T v = rng.unit();
        const T z = T(2) * u - T(1);
        const T r = sqrt(T(1) - z * z);
        if constexpr (EXACT) {
            const double phi = 2 * kPi * v;
            return V3<T>{c.x + R * r * cos(phi), c.y + R * r * sin(phi), c.z + R * z};
        }
        T s, co;
        sincos_2pi<T>(v, s, co);
        return V3<T>{c.x + R * r * co, c.y + R * r * s, c.z + R * z};
    }
}

// Uniform point in the ball, src/wos.cpp:33-56.
template <int DIM, bool EXACT, typename T, class Rng>
__device__ __forceinline__ V3<T> ball_sample(V3<T> c, T R, Rng &rng) {
    if (DIM == 2) {
        const T u = rng.unit();
        const T r = R * sqrt(rng.unit_open());
        if constexpr (EXACT) {
            const double theta = u * 2 * kPi;
            return V3<T>{c.x + r * cos(theta), c.y + r * sin(theta), T(0)};
        }
        T s, co;
        sincos_2pi<T>(u, s, co);
        return V3<T>{c.x + r * co, c.y + r * s, T(0)};
    } else {
        const T u = rng.unit();
        const T v = rng.unit();
        const T w = rng.unit_open();
        const T z = T(2) * u - T(1);
        const T surf = sqrt(T(1) - z * z);
        const T vol = R * cbrt(w);
        if constexpr (EXACT) {
            const double phi = 2 * kPi * v;
            return V3<T>{c.x + vol * surf * cos(phi), c.y + vol * surf * sin(phi),
                         c.z + vol * z};
        }
        T s, co;
        sincos_2pi<T>(v, s, co);
        return V3<T>{c.x + vol * surf * co, c.y + vol * surf * s, c.z + vol * z};
    }
}

// Point at `radius` from c in a uniform direction (the angular part of the
// Green samplers, src/equations/poisson.cpp:62-72 / :105-117).
template <int DIM, bool EXACT, typename T, class Rng>
__device__ __forceinline__ V3<T> direction_at(V3<T> c, T radius, Rng &rng) {
    if (DIM == 2) {
        const T u = rng.unit();
        if constexpr (EXACT) {
            const double angle = 2.0 * kPi * u;
            return V3<T>{c.x + radius * cos(angle), c.y + radius * sin(angle), T(0)};
        }
        T s, co;
        sincos_2pi<T>(u, s, co);
        return V3<T>{c.x + radius * co, c.y + radius * s, T(0)};
    } else {
        const T z = T(2) * rng.unit() - T(1);
        const T u = rng.unit();
        const T xy = sqrt(T(1) - z * z);
        if constexpr (EXACT) {
            const double angle = 2.0 * kPi * u;
            return V3<T>{c.x + radius * xy * cos(angle), c.y + radius * xy * sin(angle),
                         c.z + radius * z};
        }
        T s, co;
        sincos_2pi<T>(u, s, co);
        return V3<T>{c.x + radius * xy * co, c.y + radius * xy * s, c.z + radius * z};
    }
}

// ------------------------------------------------------------ Green kernels

// include/wos/poisson.hpp:14-20, 22-24, 29-32, 34-41, 43-45, 47-51
template <typename T>
__device__ __forceinline__ T pg_green_2d(T R, T r) {
    if (!(r > T(0)) || r > R || R <= T(0)) return T(NAN);
    if (r == R) return T(0);
    return log(R / r) / (T(2) * T(kPi));
}
template <typename T>
__device__ __forceinline__ T pg_mass_2d(T R) { return R * R / T(4); }
template <typename T, class Rng>
__device__ __forceinline__ T pg_sample_radius_2d(T R, Rng &rng) {
    const T u = rng.unit_open();
    const T v = rng.unit_open();
    return R * sqrt(u * v);
}
template <typename T>
__device__ __forceinline__ T pg_green_3d(T R, T r) {
    if (!(r > T(0)) || r > R || R <= T(0)) return T(NAN);
    if (r == R) return T(0);
    return (R - r) / (T(4) * T(kPi) * r * R);
}
template <typename T>
__device__ __forceinline__ T pg_mass_3d(T R) { return R * R / T(6); }
template <typename T, class Rng>
__device__ __forceinline__ T pg_sample_radius_3d(T R, Rng &rng) {
    T u = rng.unit_open(), v = rng.unit_open();
    const T a = -log(u * v);
    u = rng.unit_open();
    v = rng.unit_open();
    const T b = -log(u * v);
    return R * a / (a + b);
}

// include/wos/screened.hpp:14-89
template <typename T>
__device__ __forceinline__ T sc_weight_2d(T alpha, T R) {
    const T x = alpha * R;
    if (x == T(0)) return T(1);
    if (x < T(1e-3)) {
        const T x2 = x * x;
        return T(1) - x2 / T(4) + T(3) * x2 * x2 / T(64);
    }
    return exp(-log_i0(x));
}
template <typename T>
__device__ __forceinline__ T sc_green_2d(T alpha, T R, T r) {
    if (!(r > T(0)) || r > R || R <= T(0)) return T(NAN);
    if (r == R) return T(0);
    const T x = alpha * r, X = alpha * R;
    if (X < T(1e-5)) return pg_green_2d(R, r);
    const T la = log_k0(x);
    const T lb = log_i0(x) + log_k0(X) - log_i0(X);
    T delta = lb - la;
    if (delta > T(0)) delta = T(0);
    return exp(la) * (-expm1(delta)) / (T(2) * T(kPi));
}
template <typename T>
__device__ __forceinline__ T sc_mass_2d(T alpha, T R) {
    const T x = alpha * R;
    if (x < T(1e-3)) {
        const T x2 = x * x;
        return R * R * (T(1) / T(4) - T(3) * x2 / T(64) + T(19) * x2 * x2 / T(2304));
    }
    return -expm1(-log_i0(x)) / (alpha * alpha);
}
template <typename T>
__device__ __forceinline__ T sc_weight_3d(T alpha, T R) {
    const T x = alpha * R;
    if (x == T(0)) return T(1);
    if (x < T(1e-3)) {
        const T x2 = x * x;
        return T(1) - x2 / T(6) + T(7) * x2 * x2 / T(360);
    }
    return T(2) * x * exp(-x) / (-expm1(T(-2) * x));
}
template <typename T>
__device__ __forceinline__ T sc_green_3d(T alpha, T R, T r) {
    if (!(r > T(0)) || r > R || R <= T(0)) return T(NAN);
    if (r == R) return T(0);
    const T x = alpha * r, X = alpha * R;
    if (X < T(1e-5)) return pg_green_3d(R, r);
    const T ratio = exp(-x) * (-expm1(T(-2) * (X - x))) / (-expm1(T(-2) * X));
    return ratio / (T(4) * T(kPi) * r);
}
template <typename T>
__device__ __forceinline__ T sc_mass_3d(T alpha, T R) {
    const T x = alpha * R;
    if (x < T(1e-3)) {
        const T x2 = x * x;
        return R * R * (T(1) / T(6) - T(7) * x2 / T(360) + T(31) * x2 * x2 / T(15120));
    }
    return (T(1) - sc_weight_3d(alpha, R)) / (alpha * alpha);
}
template <typename T>
__device__ __forceinline__ T clamp_probability(T v) {
    const T lo = (v < T(1)) ? v : T(1);
    return (T(0) < lo) ? lo : T(0);
}
template <typename T, class Rng>
__device__ __forceinline__ T sc_normal(Rng &rng) {
    const T radius = sqrt(T(-2) * log(rng.unit_open()));
    const T angle_u = rng.unit();
    return radius * cos(T(2) * T(kPi) * angle_u);
}

// Rejection samplers of the screened Green radius (screened.hpp:103-156).
// The reference loops until acceptance; here the loop is capped and the cap
// raises `overflow` (acceptance rates are ~0.5 or higher, so 4096 proposals
// are never used up in practice).
constexpr int kRejectionCap = 4096;

template <typename T, class Rng>
__device__ __forceinline__ T sc_sample_radius_2d(T alpha, T R, Rng &rng, bool &overflow) {
    const T X = alpha * R;
    T r = R * T(0.5);
    for (int it = 0; it < kRejectionCap; ++it) {
        T acc;
        if (X < T(2)) {
            r = pg_sample_radius_2d(R, rng);
            const T proposal = pg_green_2d(R, r);
            acc = sc_green_2d(alpha, R, r) / proposal;
        } else {
            const T time = -log(rng.unit_open()) / (alpha * alpha);
            r = sqrt(T(-4) * time * log(rng.unit_open()));
            if (r >= R) continue;
            const T x = alpha * r;
            const T lr = log_i0(x) + log_k0(X) - log_i0(X) - log_k0(x);
            acc = -expm1((lr < T(0)) ? lr : T(0));
        }
        if (rng.unit() < clamp_probability(acc)) return r;
    }
    overflow = true;
    return r;
}

template <typename T, class Rng>
__device__ __forceinline__ T sc_sample_radius_3d(T alpha, T R, Rng &rng, bool &overflow) {
    const T X = alpha * R;
    T r = R * T(0.5);
    for (int it = 0; it < kRejectionCap; ++it) {
        T acc;
        if (X < T(2)) {
            r = pg_sample_radius_3d(R, rng);
            const T proposal = pg_green_3d(R, r);
            acc = sc_green_3d(alpha, R, r) / proposal;
        } else {
            const T time = -log(rng.unit_open()) / (alpha * alpha);
            const T scale = sqrt(T(2) * time);
            const T x0 = scale * sc_normal<T>(rng);
            const T x1 = scale * sc_normal<T>(rng);
            const T x2 = scale * sc_normal<T>(rng);
            r = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
            if (r >= R) continue;
            const T x = alpha * r;
            acc = (-expm1(T(-2) * (X - x))) / (-expm1(T(-2) * X));
        }
        if (rng.unit() < clamp_probability(acc)) return r;
    }
    overflow = true;
    return r;
}

// ---------------------------------------------------------------- equations

// Volume of the ball (include/wos/wos.hpp:21-27).
template <int DIM, typename T>
__device__ __forceinline__ T ball_volume(T R) {
    if (DIM == 2) return T(kPi) * R * R;
    const T rc = R * R * R;
    return T(4) * T(kPi) * rc / T(3);
}

// laplace (src/equations/laplace.cpp:12-43)
template <int DIM>
struct Laplace {
    static constexpr bool kSource = false, kScreening = false;
    template <typename T>
    __device__ T boundary(V3<T> p, int bid) const {
        if (DIM == 2) return bid == 0 ? p.x * p.x - p.y * p.y : T(0);
        return harmonic_y5(p.x, p.y, p.z);
    }
    template <typename T>
    __device__ T screening(T) const { return T(1); }
};

// poisson (src/equations/poisson.cpp:15-118): 2D uniform load f = 0.1 on the
// disk of radius 0.15 at the origin with g = 0; 3D f = 0 (draws still
// consumed) with the degree-5 harmonic boundary data.
template <int DIM>
struct Poisson {
    static constexpr bool kSource = true, kScreening = false;
    int mode;
    double alpha;
    template <typename T>
    __device__ T boundary(V3<T> p, int) const {
        if (DIM == 2) return T(0);
        return harmonic_y5(p.x, p.y, p.z);
    }
    template <typename T>
    __device__ bool may_intersect(V3<T> c, T R) const {
        const T dx = c.x - T(0), dy = c.y - T(0);
        const T reach = R + T(0.15);
        return dx * dx + dy * dy <= reach * reach;
    }
    template <typename T>
    __device__ T source(V3<T> p) const {
        if (DIM == 3) return T(0);
        const T dx = p.x - T(0), dy = p.y - T(0);
        return dx * dx + dy * dy <= T(0.15) * T(0.15) ? T(0.1) : T(0);
    }
    template <typename T>
    __device__ T green(T R, T r) const {
        return DIM == 2 ? pg_green_2d(R, r) : pg_green_3d(R, r);
    }
    template <typename T>
    __device__ T green_mass(T R) const {
        return DIM == 2 ? pg_mass_2d(R) : pg_mass_3d(R);
    }
    template <typename T, class Rng>
    __device__ T green_radius(T R, Rng &rng, bool &) const {
        return DIM == 2 ? pg_sample_radius_2d(R, rng) : pg_sample_radius_3d(R, rng);
    }
    template <typename T>
    __device__ T screening(T) const { return T(1); }
};

// screened_poisson (src/equations/screened_poisson.cpp:40-141): 2D bump f = 5
// on the disk of radius 0.5 at (0.45, 0), g = x^2 - y^2 on boundary 0,
// weight 1/I0(alpha R); 3D has no source (weight alpha R / sinh(alpha R) only)
// and the degree-5 harmonic boundary data.
template <int DIM>
struct Screened {
    static constexpr bool kSource = (DIM == 2), kScreening = true;
    int mode;
    double alpha;
    template <typename T>
    __device__ T boundary(V3<T> p, int bid) const {
        if (DIM == 2) return bid == 0 ? p.x * p.x - p.y * p.y : T(0);
        return harmonic_y5(p.x, p.y, p.z);
    }
    template <typename T>
    __device__ bool may_intersect(V3<T> c, T R) const {
        const T dx = c.x - T(0.45), dy = c.y - T(0);
        const T reach = R + T(0.5);
        return dx * dx + dy * dy <= reach * reach;
    }
    template <typename T>
    __device__ T source(V3<T> p) const {
        if (DIM == 3) return T(0);
        return sqrt((p.x - T(0.45)) * (p.x - T(0.45)) + p.y * p.y) <= T(0.5) ? T(5) : T(0);
    }
    template <typename T>
    __device__ T green(T R, T r) const {
        const T a = static_cast<T>(alpha);
        return DIM == 2 ? sc_green_2d(a, R, r) : sc_green_3d(a, R, r);
    }
    template <typename T>
    __device__ T green_mass(T R) const {
        const T a = static_cast<T>(alpha);
        return DIM == 2 ? sc_mass_2d(a, R) : sc_mass_3d(a, R);
    }
    template <typename T, class Rng>
    __device__ T green_radius(T R, Rng &rng, bool &overflow) const {
        const T a = static_cast<T>(alpha);
        return DIM == 2 ? sc_sample_radius_2d(a, R, rng, overflow)
                        : sc_sample_radius_3d(a, R, rng, overflow);
    }
    template <typename T>
    __device__ T screening(T R) const {
        const T a = static_cast<T>(alpha);
        return DIM == 2 ? sc_weight_2d(a, R) : sc_weight_3d(a, R);
    }
};

// helmholtz (src/equations/helmholtz.cpp:15-78), k = 1, g = 1, no source:
// weight 1/J0(kR) in 2D and kR/sin(kR) in 3D.
template <int DIM>
struct Helmholtz {
    static constexpr bool kSource = false, kScreening = true;
    template <typename T>
    __device__ T boundary(V3<T>, int) const { return T(1); }
    template <typename T>
    __device__ T screening(T R) const {
        const T prod = R * T(1);
        if (prod < T(1e-8)) return T(1);
        return DIM == 2 ? T(1) / bessel_j0(prod) : prod / sin(prod);
    }
};

// One implicit-Euler step of the reference's transient plate problems:
// screened Poisson with alpha = 1/sqrt(kappa dt), zero boundary data and a
// source built from the previous step's grid field u_prev, read by the
// reference's FieldSampler2D (apps/welding/include/welding/field_sampler.hpp:
// 32-126).  Sources, by `kind`:
//   0  alpha^2 u_prev                       cooling (apps/welding/src/level0_cooling.cpp:194-196)
//   2  alpha^2 max(0, u_prev) + fraction q_v / k   stationary Gaussian
//      (level2_transient_heat.cpp:251-259, q_v from gaussian_heat_source.hpp:38-41)
//   3  alpha^2 max(0, u_prev) + q_m / k     moving Gaussian, two Gauss-Legendre
//      components per step (level3_moving_heat.cpp:189-194,
//      moving_gaussian_heat_source.hpp:73-88)
// Expression order follows the reference (the exact path rounds like it).
struct TransientDesc {
    double alpha;
    double fraction;       // kind 2: share of the step with the heat source on
    double conductivity;
    double power;          // kind 2: absorbed power
    double thickness, ix, iy;  // kind 2: plate thickness, Gaussian integrals over x and y
    double cx, cy, sx, sy;     // kind 2: centre and widths
    int kind;
    int moving;            // kind 3: 2 when the source is on during the step, else 0
    double mx[2], my[2], mcoef[2];  // kind 3: component centres and coefficients
    const double *prev;    // previous field, (i, j) row-major, nx * ny
    int nx, ny;
    double xmin, xmax, ymin, ymax;
    int cubic;             // 1: cubic Lagrange history interpolation, 0: bilinear
    int pad;
};

__device__ __forceinline__ double clamp_ref(double v, double lo, double hi) {
    return v < lo ? lo : (hi < v ? hi : v);  // std::clamp
}

__device__ __forceinline__ double field_at(const TransientDesc &t, int i, int j) {
    return t.prev[static_cast<long long>(i) * t.ny + j];
}

__device__ __forceinline__ void cubic_weights(double c, double w[4]) {
    w[0] = -(c - 1.0) * (c - 2.0) * (c - 3.0) / 6.0;
    w[1] = c * (c - 2.0) * (c - 3.0) / 2.0;
    w[2] = -c * (c - 1.0) * (c - 3.0) / 2.0;
    w[3] = c * (c - 1.0) * (c - 2.0) / 6.0;
}

// FieldSampler2D::sample
__device__ __forceinline__ double field_sample(const TransientDesc &t, double x, double y) {
    const double gx = clamp_ref((x - t.xmin) / (t.xmax - t.xmin) * static_cast<double>(t.nx - 1),
                                0.0, static_cast<double>(t.nx - 1));
    const double gy = clamp_ref((y - t.ymin) / (t.ymax - t.ymin) * static_cast<double>(t.ny - 1),
                                0.0, static_cast<double>(t.ny - 1));
    if (t.cubic && t.nx >= 4 && t.ny >= 4) {
        int ix = static_cast<int>(floor(gx)) - 1;
        int iy = static_cast<int>(floor(gy)) - 1;
        ix = ix < 0 ? 0 : (t.nx - 4 < ix ? t.nx - 4 : ix);
        iy = iy < 0 ? 0 : (t.ny - 4 < iy ? t.ny - 4 : iy);
        double wx[4], wy[4];
        cubic_weights(gx - static_cast<double>(ix), wx);
        cubic_weights(gy - static_cast<double>(iy), wy);
        double value = 0.0;
        for (int di = 0; di < 4; ++di) {
            double row = 0.0;
            for (int dj = 0; dj < 4; ++dj) row += wy[dj] * field_at(t, ix + di, iy + dj);
            value += wx[di] * row;
        }
        return value;
    }
    const int i0 = static_cast<int>(floor(gx));
    const int j0 = static_cast<int>(floor(gy));
    const int i1 = i0 + 1 < t.nx - 1 ? i0 + 1 : t.nx - 1;
    const int j1 = j0 + 1 < t.ny - 1 ? j0 + 1 : t.ny - 1;
    const double tx = gx - static_cast<double>(i0);
    const double ty = gy - static_cast<double>(j0);
    const double v00 = field_at(t, i0, j0);
    const double v10 = field_at(t, i1, j0);
    const double v01 = field_at(t, i0, j1);
    const double v11 = field_at(t, i1, j1);
    const double lower = (1.0 - tx) * v00 + tx * v10;
    const double upper = (1.0 - tx) * v01 + tx * v11;
    return (1.0 - ty) * lower + ty * upper;
}

// The equations' source(point)
__device__ __forceinline__ double transient_source(const TransientDesc &t, double x, double y) {
    const double v = field_sample(t, x, y);
    if (t.kind == 0) return t.alpha * t.alpha * v;
    const double previous = t.alpha * t.alpha * (0.0 < v ? v : 0.0);
    if (t.kind == 3) {
        double value = 0.0;
        for (int k = 0; k < t.moving; ++k) {
            const double dx = (x - t.mx[k]) / t.sx;
            const double dy = (y - t.my[k]) / t.sy;
            value += t.mcoef[k] * exp(-0.5 * (dx * dx + dy * dy));
        }
        return previous + value / t.conductivity;
    }
    double heat = 0.0;
    if (t.fraction > 0.0) {
        const double dx = (x - t.cx) / t.sx;
        const double dy = (y - t.cy) / t.sy;
        const double shape = exp(-0.5 * (dx * dx + dy * dy));
        const double density = t.power * shape / (t.thickness * t.ix * t.iy);
        heat = t.fraction * density / t.conductivity;
    }
    return previous + heat;
}

template <int DIM>
struct Transient {
    static constexpr bool kSource = true, kScreening = true;
    int mode;  // always kGreen: screened Green source samples
    double alpha;
    const TransientDesc *t;
    template <typename T>
    __device__ T boundary(V3<T>, int) const { return T(0); }
    template <typename T>
    __device__ bool may_intersect(V3<T>, T) const { return true; }
    template <typename T>
    __device__ T source(V3<T> p) const {
        return static_cast<T>(transient_source(*t, static_cast<double>(p.x),
                                               static_cast<double>(p.y)));
    }
    template <typename T>
    __device__ T green(T R, T r) const { return sc_green_2d(static_cast<T>(alpha), R, r); }
    template <typename T>
    __device__ T green_mass(T R) const { return sc_mass_2d(static_cast<T>(alpha), R); }
    template <typename T, class Rng>
    __device__ T green_radius(T R, Rng &rng, bool &overflow) const {
        return sc_sample_radius_2d(static_cast<T>(alpha), R, rng, overflow);
    }
    template <typename T>
    __device__ T screening(T R) const { return sc_weight_2d(static_cast<T>(alpha), R); }
};

// Stationary plate heating, the reference's welding level 1
// (apps/welding/src/level1_stationary_heat.cpp:75-191): -Lap u = f on the
// plate [xmin, xmax] x [ymin, ymax] with u = 0 on its edges.  Sources, by
// `kind`:
//   0  manufactured: lambda * peak sin(pi x / Lx) sin(pi y / Ly) with
//      lambda = pi^2 (1/Lx^2 + 1/Ly^2) (ManufacturedPoisson2D, :75-103)
//   1  Gaussian: q_v / k, q_v the finite-plate Gaussian
//      (StationaryGaussianHeat2D, :132-191; gaussian_heat_source.hpp:38-41)
// The Gaussian also supplies the Green-source MIS proposal: the finite-plate
// Gaussian drawn by rejection from the untruncated normal
// (gaussian_heat_source.hpp:54-73), density shape / (ix iy) on the plate
// (:45-51).  Expression order follows the reference.
struct PlateDesc {
    int kind;
    int max_attempts;          // proposal rejection cap (1e6 in the reference)
    double peak, length_x, length_y, eigen;            // kind 0
    double power, thickness, conductivity, ix, iy;     // kind 1
    double cx, cy, sx, sy;
    double beta;               // MIS: probability of a Green sample
    double xmin, xmax, ymin, ymax;
};

__device__ __forceinline__ double plate_shape(const PlateDesc &d, double x, double y) {
    const double dx = (x - d.cx) / d.sx;
    const double dy = (y - d.cy) / d.sy;
    return exp(-0.5 * (dx * dx + dy * dy));
}

__device__ __forceinline__ double plate_source(const PlateDesc &d, double x, double y) {
    if (d.kind == 0) {
        const double exact = d.peak * sin(kPi * x / d.length_x) * sin(kPi * y / d.length_y);
        return d.eigen * exact;
    }
    const double density = d.power * plate_shape(d, x, y) / (d.thickness * d.ix * d.iy);
    return density / d.conductivity;
}

template <int DIM>
struct Plate {
    static constexpr bool kSource = true, kScreening = false, kProposal = true;
    int mode;  // kGreen, kUniform or (Gaussian only) kMis
    PlateDesc d;
    template <typename T>
    __device__ T boundary(V3<T>, int) const { return T(0); }
    template <typename T>
    __device__ bool may_intersect(V3<T>, T) const { return true; }
    template <typename T>
    __device__ T source(V3<T> p) const {
        return static_cast<T>(
            plate_source(d, static_cast<double>(p.x), static_cast<double>(p.y)));
    }
    template <typename T>
    __device__ T green(T R, T r) const { return pg_green_2d(R, r); }
    template <typename T>
    __device__ T green_mass(T R) const { return pg_mass_2d(R); }
    template <typename T, class Rng>
    __device__ T green_radius(T R, Rng &rng, bool &) const {
        return pg_sample_radius_2d(R, rng);
    }
    template <typename T>
    __device__ T screening(T) const { return T(1); }
    __device__ double mis_green_probability() const { return d.beta; }
    __device__ double proposal_pdf(double x, double y) const {
        if (x < d.xmin || x > d.xmax || y < d.ymin || y > d.ymax) return 0.0;
        return plate_shape(d, x, y) / (d.ix * d.iy);
    }
    // GaussianHeatSource2D::sample_spatial_distribution; sets `overflow`
    // when every one of the max_attempts proposals fell off the plate.
    template <bool EXACT, class Rng>
    __device__ V3<double> proposal_sample(Rng &rng, bool &overflow) const {
        constexpr double two_pi = 2.0 * kPi;
        for (int attempt = 0; attempt < d.max_attempts; ++attempt) {
            const double magnitude = sqrt(-2.0 * log(rng.unit64_open()));
            const double u = rng.unit64();
            double s, c;
            if constexpr (EXACT) {
                const double angle = two_pi * u;
                c = cos(angle);
                s = sin(angle);
            } else {
                sincospi(2.0 * u, &s, &c);
            }
            const V3<double> q{d.cx + d.sx * magnitude * c, d.cy + d.sy * magnitude * s, 0.0};
            if (q.x >= d.xmin && q.x <= d.xmax && q.y >= d.ymin && q.y <= d.ymax) return q;
        }
        overflow = true;
        return V3<double>{d.cx, d.cy, 0.0};
    }
};

// Equations that carry a source proposal (kProposal) can run Green-source MIS.
template <class Eq, class = void>
struct HasProposal {
    static constexpr bool value = false;
};
template <class Eq>
struct HasProposal<Eq, decltype(void(Eq::kProposal))> {
    static constexpr bool value = Eq::kProposal;
};

// One ball's Green-source MIS estimate with the balance heuristic over a
// random mixture (include/wos/source_sampling.hpp:35-78): a Green sample
// with probability beta, else a proposal sample; samples outside the ball
// count zero.  The distances, densities and source are evaluated in FP64.
template <int DIM, bool EXACT, typename T, class Eq, class Rng>
__device__ __forceinline__ double mis_contribution(const Eq &eq, V3<T> p, T R, Rng &rng,
                                                   bool &overflow) {
    const double beta = eq.mis_green_probability();
    V3<double> y;
    if (static_cast<double>(rng.unit()) < beta) {
        const T radius = eq.green_radius(R, rng, overflow);
        const V3<T> g = direction_at<DIM, EXACT, T>(p, radius, rng);
        y = V3<double>{static_cast<double>(g.x), static_cast<double>(g.y), 0.0};
    } else {
        y = eq.template proposal_sample<EXACT>(rng, overflow);
    }
    const V3<double> c{static_cast<double>(p.x), static_cast<double>(p.y), 0.0};
    const double Rd = static_cast<double>(R);
    const double distance = dist<DIM>(c, y);
    if (!(distance > 0.0 && distance < Rd)) return 0.0;
    const double green_mass = pg_mass_2d(Rd);
    const double green_value = pg_green_2d(Rd, distance);
    const double green_pdf = green_value / green_mass;
    const double source_pdf = eq.proposal_pdf(y.x, y.y);
    const double mixture_pdf = beta * green_pdf + (1.0 - beta) * source_pdf;
    if (!(mixture_pdf > 0.0)) return 0.0;
    const double source_value = eq.source(y);
    return source_value == 0.0 ? 0.0 : green_value * source_value / mixture_pdf;
}

// One iteration of the walk loop body before the closest-point query
// (include/wos/wos.hpp:69-115): the source contribution of the current ball,
// the screening weight, then the step to the sphere.  Returns the new point.
template <int DIM, bool EXACT, typename T, class Eq, class WalkRng, class SrcRng>
__device__ __forceinline__ V3<T> walk_body(const Eq &eq, V3<T> p, T R, T &sample, T &weight,
                                           WalkRng &walk, SrcRng &src, bool &overflow) {
    if constexpr (Eq::kSource) {
        bool may = true;
        if (DIM == 2) may = eq.may_intersect(p, R);
        bool mis = false;
        if constexpr (HasProposal<Eq>::value) {
            if (may && eq.mode == kMis) {
                sample += weight * static_cast<T>(
                                       mis_contribution<DIM, EXACT, T>(eq, p, R, src, overflow));
                mis = true;
            }
        }
        if (may && !mis) {
            if (eq.mode == kGreen) {
                const T radius = eq.green_radius(R, src, overflow);
                const V3<T> sp = direction_at<DIM, EXACT, T>(p, radius, src);
                const T f = eq.source(sp);
                if (f != T(0)) sample += weight * eq.green_mass(R) * f;
            } else {
                const V3<T> sp = ball_sample<DIM, EXACT, T>(p, R, src);
                const T f = eq.source(sp);
                if (f != T(0)) {
                    sample += weight * ball_volume<DIM, T>(R) * f * eq.green(R, dist<DIM>(p, sp));
                }
            }
        }
    }
    if constexpr (Eq::kScreening) weight *= eq.screening(R);
    return sphere_step<DIM, EXACT, T>(p, R, walk);
}

}  // namespace wosb
