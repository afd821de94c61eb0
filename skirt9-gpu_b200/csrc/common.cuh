// Shared device helpers of the sm_100a photon-packet tracer: exact FP64 arithmetic without FMA
// contraction (used where results must match the reference CPU generators bit for bit), the
// Philox4x32-10 counter-based generator (one stream per history index), and the small sampling
// routines of the life cycle.
#pragma once

#include <cstdint>
#include <cfloat>
#include <cmath>

#define SKG_HD __host__ __device__ __forceinline__
#define SKG_D __device__ __forceinline__

namespace skg {

// ---------------------------------------------------------------------------------------------
// Exact IEEE double operations. The reference is compiled for x86-64 with SSE2 (no FMA), so
// every multiply and add is rounded separately; __dmul_rn/__dadd_rn are never fused by nvcc.
// ---------------------------------------------------------------------------------------------
SKG_D double xmul(double a, double b) { return __dmul_rn(a, b); }
SKG_D double xadd(double a, double b) { return __dadd_rn(a, b); }
SKG_D double xsub(double a, double b) { return __dsub_rn(a, b); }
// a*b + c*d + e*f evaluated left to right with separate roundings (Vec::dot, SKIRT/utils/Vec.hpp:70)
SKG_D double xdot3(double a, double b, double c, double d, double e, double f)
{
    return xadd(xadd(xmul(a, b), xmul(c, d)), xmul(e, f));
}

// The IEEE quotient a / b from y = 1 / b rounded to nearest (computed once per ray): q = a * y is
// within one ulp of a / b, the FMA residual r = a - b * q is exact, and q + r * y rounded once is
// the correctly rounded quotient (Markstein, IBM J. Res. Dev. 34 (1990) 111-119; the division
// theorem of Muller et al., Handbook of Floating-Point Arithmetic, 2018, section 4.9) for finite
// operands whose quotient neither overflows nor underflows: three FP64 operations instead of a
// division per wall distance.
SKG_D double qdiv(double a, double b, double y)
{
    double q = __dmul_rn(a, y);
    double r = __fma_rn(-q, b, a);
    return __fma_rn(r, y, q);
}

// ---------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror & Shaw 2011, "Parallel random numbers: as easy as 1, 2, 3").
// Each history draws from its own counter stream: key = seed, counter = (draw, 0, hist_lo, hist_hi).
// ---------------------------------------------------------------------------------------------
struct U4 { uint32_t x, y, z, w; };

SKG_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo)
{
    uint64_t p = static_cast<uint64_t>(a) * static_cast<uint64_t>(b);
    hi = static_cast<uint32_t>(p >> 32);
    lo = static_cast<uint32_t>(p);
}

SKG_HD U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
    for (int r = 0; r < 10; ++r)
    {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(M0, c.x, hi0, lo0);
        mulhilo32(M1, c.z, hi1, lo1);
        U4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// uniform deviate in the open interval (0,1) from 52 random bits: (j + 1/2) * 2^-52
SKG_HD double u01_from_bits(uint32_t hi, uint32_t lo)
{
    uint64_t j = ((static_cast<uint64_t>(hi) << 32) | lo) >> 12;  // 52 bits
    return (static_cast<double>(j) + 0.5) * 2.220446049250313080847e-16;
}

struct Rng
{
    uint32_t k0, k1;     // key (seed)
    uint32_t c2, c3;     // history index
    uint32_t ctr;        // draw block counter
    int hasSpare;
    double spare;

    SKG_HD void start(uint64_t seed, uint64_t history)
    {
        k0 = static_cast<uint32_t>(seed);
        k1 = static_cast<uint32_t>(seed >> 32);
        c2 = static_cast<uint32_t>(history);
        c3 = static_cast<uint32_t>(history >> 32);
        ctr = 0;
        hasSpare = 0;
        spare = 0.;
    }
    SKG_HD double uniform()
    {
        if (hasSpare)
        {
            hasSpare = 0;
            return spare;
        }
        U4 c{ctr++, 0u, c2, c3};
        U4 r = philox4x32_10(c, k0, k1);
        spare = u01_from_bits(r.z, r.w);
        hasSpare = 1;
        return u01_from_bits(r.x, r.y);
    }
};

// ---------------------------------------------------------------------------------------------
// Sampling helpers (restated from SKIRT/core/Random.cpp and DustMix.cpp)
// ---------------------------------------------------------------------------------------------

// Random::direction() (Random.cpp:121-128) with Direction(theta, phi) (Direction.cpp:11-37)
SKG_D void isotropicDirection(Rng& rng, double& kx, double& ky, double& kz)
{
    double theta = acos(2.0 * rng.uniform() - 1.0);
    double phi = 2.0 * M_PI * rng.uniform();
    const double eps = 1e-8;
    if (theta <= eps)
    {
        kx = 0.; ky = 0.; kz = 1.;
    }
    else if (theta >= M_PI - eps)
    {
        kx = 0.; ky = 0.; kz = -1.;
    }
    else
    {
        double st = sin(theta);
        kx = st * cos(phi);
        ky = st * sin(phi);
        kz = cos(theta);
    }
}

// Random::direction(bfk, costheta) (Random.cpp:130-163): rotate about the old direction
SKG_D void rotateDirection(Rng& rng, double costheta, double& kx, double& ky, double& kz)
{
    double phi = 2.0 * M_PI * rng.uniform();
    double cosphi = cos(phi);
    double sinphi = sin(phi);
    double sintheta = sqrt(fabs((1.0 - costheta) * (1.0 + costheta)));
    double nx, ny, nz;
    if (kz > 0.99999)
    {
        nx = cosphi * sintheta;
        ny = sinphi * sintheta;
        nz = costheta;
    }
    else if (kz < -0.99999)
    {
        nx = cosphi * sintheta;
        ny = sinphi * sintheta;
        nz = -costheta;
    }
    else
    {
        double root = sqrt((1.0 - kz) * (1.0 + kz));
        nx = sintheta / root * (-kx * kz * cosphi + ky * sinphi) + kx * costheta;
        ny = -sintheta / root * (ky * kz * cosphi + kx * sinphi) + ky * costheta;
        nz = root * sintheta * cosphi + kz * costheta;
    }
    kx = nx;
    ky = ny;
    kz = nz;
}

// Random::exponCutoff (Random.cpp:105-121): exponential deviate truncated at xmax, by rejection
SKG_D double exponCutoff(Rng& rng, double xmax)
{
    if (xmax == 0.0) return 0.0;
    if (xmax < 1e-10) return rng.uniform() * xmax;
    double c = 1.0 - exp(-xmax);
    for (int guard = 0; guard < 64; ++guard)
    {
        double x = -log(1.0 - rng.uniform() * c);
        if (x <= xmax) return x;
    }
    return xmax;
}

// Henyey-Greenstein phase function value and its 4-degree average for |g| > 0.95 (DustMix.cpp:395-428)
SKG_D double valueHG(double g, double costheta)
{
    double t = 1. + g * g - 2. * g * costheta;
    return (1. - g) * (1. + g) / sqrt(t * t * t);
}
SKG_D double integralHG(double g, double cosalpha, double cosbeta)
{
    double ta = sqrt(1. + g * g - 2. * g * cosalpha);
    double tb = sqrt(1. + g * g - 2. * g * cosbeta);
    double f1 = (1. - g) * (1. + g) / g;
    double f2 = (tb - ta) / (tb * ta);
    return f1 * f2;
}
SKG_D double meanHG(double g, double costheta)
{
    const double delta = 4. * M_PI / 180.;
    double theta = acos(fmin(1., fmax(-1., costheta)));
    double cosalpha = cos(theta - delta);
    double cosbeta = cos(theta + delta);
    if (theta < delta)
        return (integralHG(g, 1., cosalpha) + integralHG(g, 1., cosbeta)) / (2. - cosalpha - cosbeta);
    if (theta > M_PI - delta)
        return (integralHG(g, cosalpha, -1.) + integralHG(g, cosbeta, -1.)) / (2. + cosalpha + cosbeta);
    return integralHG(g, cosalpha, cosbeta) / (cosalpha - cosbeta);
}
SKG_D double phaseHG(double g, double costheta)
{
    return fabs(g) > 0.95 ? meanHG(g, costheta) : valueHG(g, costheta);
}

// SpecialFunctions::lnmean(x1, x2, lnx1, lnx2) (SKIRT/utils/SpecialFunctions.cpp:860-880),
// in the precision of the walk accumulators
template<typename R>
SKG_D R lnmean4(R x1, R x2, R lnx1, R lnx2)
{
    if (x1 > x2)
    {
        R t = x1; x1 = x2; x2 = t;
        t = lnx1; lnx1 = lnx2; lnx2 = t;
    }
    if (x1 <= R(0)) return R(0);
    R x = x2 / x1 - R(1);
    if (x < R(1e-3))
        return x1 / (R(1) - R(1) / R(2) * x + R(1) / R(3) * x * x - R(1) / R(4) * x * x * x + R(1) / R(5) * x * x * x * x
                     - R(1) / R(6) * x * x * x * x * x);
    return (x2 - x1) / (lnx2 - lnx1);
}

// NR::locateClip on an ascending border array of n entries (SKIRT/utils/NR.hpp:177-182)
template<typename T>
SKG_HD int locateClip(const T* xv, int n, T x)
{
    if (x < xv[0]) return 0;
    int jl = -1, ju = n - 1;
    while (ju - jl > 1)
    {
        int jm = (ju + jl) >> 1;
        if (x < xv[jm])
            ju = jm;
        else
            jl = jm;
    }
    return jl;
}

// NR::locate on an ascending array of n entries (SKIRT/utils/NR.hpp:168-173): -1 below the first
// entry, n - 1 above the last, and n - 2 exactly at the last
SKG_HD int locateNR(const double* xv, int n, double x)
{
    if (x == xv[n - 1]) return n - 2;
    int jl = -1, ju = n;
    while (ju - jl > 1)
    {
        int jm = (ju + jl) >> 1;
        if (x < xv[jm])
            ju = jm;
        else
            jl = jm;
    }
    return jl;
}

// NR::clampedValue<NR::interpolateLogLog>(x, xv, yv) (SKIRT/utils/NR.hpp:349-358, 394-401): the
// table's end values outside it, power-law interpolation inside; a non-positive end value gives 0
// between the points, and a first interval starting at x = 0 (where the power law is undefined)
// gives the interval's lower value
SKG_HD double clampedLogLog(const double* xv, const double* yv, int n, double x)
{
    int i = locateNR(xv, n, x);
    if (i < 0) return yv[0];
    if (i >= n - 1) return yv[n - 1];
    double x1 = xv[i], x2 = xv[i + 1], f1 = yv[i], f2 = yv[i + 1];
    if (f1 <= 0 || f2 <= 0)
    {
        if (x == x1) return f1;
        if (x == x2) return f2;
        return 0;
    }
    if (!(x1 > 0)) return f1;
    return f1 * exp(log(x / x1) / log(x2 / x1) * (log(f2 / f1)));
}

// NR::interpolateLogLog (SKIRT/utils/NR.hpp:349-358): power-law interpolation between (x1, f1) and
// (x2, f2); a non-positive end value gives that end's value at the end points and 0 between them
SKG_HD double interpLogLog(double x, double x1, double x2, double f1, double f2)
{
    if (f1 <= 0 || f2 <= 0)
    {
        if (x == x1) return f1;
        if (x == x2) return f2;
        return 0;
    }
    return f1 * exp(log(x / x1) / log(x2 / x1) * (log(f2 / f1)));
}

// SpecialFunctions::gln(p, x) (SKIRT/utils/SpecialFunctions.cpp:798-811), the generalized
// logarithm integrating a power law in NR::cdf2
SKG_HD double gln(double p, double x)
{
    const double q = 1.0 - p;
    if (q == 0.0) return log(x);
    if (fabs(q) < 1e-3)
    {
        double lnx = log(x);
        double s = q * lnx;
        return lnx * (1.0 + 0.5 * s + 1.0 / 6.0 * s * s + 1.0 / 24.0 * s * s * s);
    }
    return (pow(x, q) - 1.0) / q;
}

// PlanckFunction(T)(lambda) (SKIRT/utils/PlanckFunction.cpp:12-27) with the constants of
// SKIRT/utils/Constants.hpp (h, c, k): 2 h c^2 / lambda^5 / (exp(h c / (k T lambda)) - 1); 0 for T = 0
SKG_HD double planckValue(double T, double lambda)
{
    const double h = 6.62606957e-34, c = 2.99792458e8, k = 1.3806488e-23;
    double f1 = h * c / (k * T);
    double f2 = 2.0 * h * c * c;
    return f2 / pow(lambda, 5) / (exp(f1 / lambda) - 1.0);
}

// std::upper_bound index on an ascending array
template<typename T>
SKG_HD int upperBound(const T* xv, int n, T x)
{
    int lo = 0, hi = n;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (x < xv[mid])
            hi = mid;
        else
            lo = mid + 1;
    }
    return lo;
}

}  // namespace skg
