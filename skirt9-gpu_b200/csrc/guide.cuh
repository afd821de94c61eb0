// Learned path guiding: a small MLP maps the state of a packet at a scattering event to a mixture
// of von Mises-Fisher lobes over the outgoing direction. Scattering then samples the composite
// density alpha * q_mix + (1 - alpha) * p_HG and multiplies the packet weight by
// p_HG / (alpha * q_mix + (1 - alpha) * p_HG), so that the estimator stays unbiased; with
// alpha = 0 the plain Henyey-Greenstein sampling of DustMix::performScattering (DustMix.cpp:490-546)
// is recovered exactly.
//
// Network: 8 inputs -> 4 hidden layers of 64 (ReLU) -> 40 outputs = 8 lobes x (logit, mu[3], kappa).
// Inputs: position / domain half size (3), incoming direction (3), log10(lambda / 0.55 um) (1),
// log(1 + tau) / 5 with tau the optical depth of the propagation path that ended here (1).
#pragma once

#include <cstdint>
#include <cmath>

#include "common.cuh"

namespace skg {

constexpr int GUIDE_IN = 8;
constexpr int GUIDE_HID = 64;
constexpr int GUIDE_LOBES = 8;
constexpr int GUIDE_OUT = 5 * GUIDE_LOBES;  // 40
constexpr int GUIDE_LAYERS = 5;
// FP32 master parameters, layer by layer: W (out x in, row-major) then b (out)
SKG_HD constexpr int guideDimIn(int l) { return l == 0 ? GUIDE_IN : GUIDE_HID; }
SKG_HD constexpr int guideDimOut(int l) { return l == GUIDE_LAYERS - 1 ? GUIDE_OUT : GUIDE_HID; }
SKG_HD constexpr int guideParamOffset(int layer)
{
    int off = 0;
    for (int l = 0; l < layer; ++l) off += guideDimOut(l) * guideDimIn(l) + guideDimOut(l);
    return off;
}
constexpr int GUIDE_NPARAMS = guideParamOffset(GUIDE_LAYERS);  // 15656
constexpr float GUIDE_KAPPA_MIN = 0.05f;
constexpr float GUIDE_KAPPA_MAX = 2000.f;
// A packet whose accumulated guiding weight ratio (product of p_HG / composite over its guided
// events) exceeds this bound scatters plainly until the ratio falls back below it. The choice
// depends on past events only, so the estimator stays unbiased, and the ratio stays below
// GUIDE_RATIO_MAX / (1 - alpha): without the bound the product over many scatterings is heavy-tailed
// and finite runs miss the rare large weights (their means come out low).
constexpr double GUIDE_RATIO_MAX = 4.0;

// one recorded scattering event of a pilot run
struct GuideRecord
{
    float f[GUIDE_IN];   // network inputs
    float k[3];          // sampled outgoing direction
    float I;             // downstream (weighted) peel-off luminosity per unit packet luminosity
    double dStart;       // the history's detected luminosity when this event's own peel-off was done
    float L;             // packet luminosity after the event
    int prev;            // previous recorded event of the same history (-1: none)
};

// network inputs of a packet at a scattering event
SKG_HD void guideFeatures(float* f, double x, double y, double z, double kx, double ky, double kz, double lambda,
                          double tau, const double* ext)
{
    double cx = 0.5 * (ext[0] + ext[3]), cy = 0.5 * (ext[1] + ext[4]), cz = 0.5 * (ext[2] + ext[5]);
    double hx = 0.5 * (ext[3] - ext[0]), hy = 0.5 * (ext[4] - ext[1]), hz = 0.5 * (ext[5] - ext[2]);
    f[0] = static_cast<float>((x - cx) / hx);
    f[1] = static_cast<float>((y - cy) / hy);
    f[2] = static_cast<float>((z - cz) / hz);
    f[3] = static_cast<float>(kx);
    f[4] = static_cast<float>(ky);
    f[5] = static_cast<float>(kz);
    f[6] = static_cast<float>(log10(lambda / 0.55e-6));
    f[7] = static_cast<float>(log1p(fmax(tau, 0.0)) / 5.0);
}

// lobe parameters from the 40 raw outputs (o[5j] logit, o[5j+1..3] direction, o[5j+4] concentration)
struct GuideMixture
{
    float logw[GUIDE_LOBES];  // log mixture weights
    float mu[GUIDE_LOBES][3];
    float kappa[GUIDE_LOBES];
};

SKG_HD float softplusf(float s) { return s > 20.f ? s : log1pf(expf(s)); }

SKG_HD void guideMixture(const float* o, GuideMixture& m)
{
    float amax = -INFINITY;
    for (int j = 0; j < GUIDE_LOBES; ++j) amax = fmaxf(amax, o[5 * j]);
    float sum = 0.f;
    for (int j = 0; j < GUIDE_LOBES; ++j) sum += expf(o[5 * j] - amax);
    float lse = amax + logf(sum);
    for (int j = 0; j < GUIDE_LOBES; ++j)
    {
        m.logw[j] = o[5 * j] - lse;
        float a = o[5 * j + 1], b = o[5 * j + 2], c = o[5 * j + 3];
        float n = sqrtf(a * a + b * b + c * c);
        if (!(n > 1e-12f))
        {
            a = 0.f; b = 0.f; c = 1.f; n = 1.f;
        }
        m.mu[j][0] = a / n;
        m.mu[j][1] = b / n;
        m.mu[j][2] = c / n;
        m.kappa[j] = fminf(softplusf(o[5 * j + 4]) + GUIDE_KAPPA_MIN, GUIDE_KAPPA_MAX);
    }
}

// log of the vMF density on the unit sphere: kappa / (2 pi (1 - e^{-2 kappa})) e^{kappa (mu.k - 1)}
SKG_HD float logVmf(float kappa, float cosang)
{
    return logf(kappa) - logf(6.283185307179586f) - log1pf(-expf(-2.f * kappa)) + kappa * (cosang - 1.f);
}

SKG_HD float guideLogDensity(const GuideMixture& m, double kx, double ky, double kz)
{
    float l[GUIDE_LOBES];
    float lmax = -INFINITY;
    for (int j = 0; j < GUIDE_LOBES; ++j)
    {
        float c = static_cast<float>(m.mu[j][0] * kx + m.mu[j][1] * ky + m.mu[j][2] * kz);
        l[j] = m.logw[j] + logVmf(m.kappa[j], fminf(1.f, fmaxf(-1.f, c)));
        lmax = fmaxf(lmax, l[j]);
    }
    float s = 0.f;
    for (int j = 0; j < GUIDE_LOBES; ++j) s += expf(l[j] - lmax);
    return lmax + logf(s);
}

// samples a direction from the mixture with three uniform deviates (lobe, cosine, azimuth);
// Wood (1994) for the vMF cosine on the 2-sphere: w = 1 + log(u + (1 - u) e^{-2 kappa}) / kappa
SKG_HD void guideSample(const GuideMixture& m, double u0, double u1, double u2, double& kx, double& ky, double& kz)
{
    int j = GUIDE_LOBES - 1;
    double acc = 0.;
    for (int i = 0; i < GUIDE_LOBES; ++i)
    {
        acc += exp(static_cast<double>(m.logw[i]));
        if (u0 < acc)
        {
            j = i;
            break;
        }
    }
    double kap = m.kappa[j];
    double w = 1.0 + log(u1 + (1.0 - u1) * exp(-2.0 * kap)) / kap;
    w = fmin(1.0, fmax(-1.0, w));
    double s = sqrt(fmax(0.0, 1.0 - w * w));
    double phi = 2.0 * M_PI * u2;
    // orthonormal frame around mu
    double mx = m.mu[j][0], my = m.mu[j][1], mz = m.mu[j][2];
    double ax, ay, az;
    if (fabs(mz) < 0.9) { ax = -my; ay = mx; az = 0.; }
    else { ax = 0.; ay = -mz; az = my; }
    double an = sqrt(ax * ax + ay * ay + az * az);
    ax /= an; ay /= an; az /= an;
    double bx = my * az - mz * ay, by = mz * ax - mx * az, bz = mx * ay - my * ax;
    double c = cos(phi) * s, d = sin(phi) * s;
    kx = w * mx + c * ax + d * bx;
    ky = w * my + c * ay + d * by;
    kz = w * mz + c * az + d * bz;
    double n = sqrt(kx * kx + ky * ky + kz * kz);
    kx /= n; ky /= n; kz /= n;
}

// Henyey-Greenstein density over solid angle (1/4pi) (1-g^2) / (1+g^2-2g cos)^{3/2}
SKG_HD double pdfHG(double g, double cosang)
{
    if (fabs(g) < 1e-6) return 1.0 / (4.0 * M_PI);
    double t = 1. + g * g - 2. * g * cosang;
    return (1. - g) * (1. + g) / (t * sqrt(t)) / (4.0 * M_PI);
}

}  // namespace skg
