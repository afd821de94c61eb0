// Per-cell dust emission of a secondary-emission segment, from the radiation field stored by the
// primary segment: the absorbed dust luminosity, the equilibrium temperature and the normalised
// emission spectrum of every cell. Compiled without FMA contraction: every sum and product is
// rounded in the reference's order, so the luminosities and temperatures equal the reference's bit
// for bit for the same radiation field (the spectra differ from it only by the last-bit differences
// of exp, log and pow).
#include "internal.hpp"

namespace skg {

namespace {

// One thread per cell m:
//  - MediumSystem::dustLuminosity (MediumSystem.cpp:2752-2762): sum over the radiation-field bins of
//    n sigma_abs(lambda_ell) J_ell in bin order (n sigma_abs is DustMix::opacityAbs, 0 for n <= 0);
//  - MediumSystem::meanIntensity (MediumSystem.cpp:2670-2680) and
//    EquilibriumDustEmissionCalculator::equilibriumTemperature (EquilibriumDustEmissionCalculator.cpp:
//    118-128): the absorbed power sum_k sigma_k (J_k + B_cmb,k) dlambda_k, summed from the last bin to
//    the first as the valarray expression's sum() does, and the temperature by linear interpolation in
//    the Planck-integrated cross sections (NR::clampedValue<NR::interpolateLinLin>, 0 without heating);
//  - the emission spectrum n sigma_abs,em(lambda) B_T(lambda) on the dust-emission grid
//    (EquilibriumDustEmissionCalculator::emissivity, DustMix::emissionSpectrum,
//    MediumSystem::dustEmissionSpectrum) and its normalised pdf and cdf on the spectrum axis xv
//    (NR::cdf<NR::interpolateLogLog> with NR::cdf2's power-law integration, SKIRT/utils/NR.hpp:494-520,
//    NR.cpp:25-53), written to the cell's row of pv / Pv.
__global__ void __launch_bounds__(256) dustCellKernel(const DustEmissionDev t, const double* __restrict__ dens,
                                                      const double* __restrict__ rf, int numCells,
                                                      const double* __restrict__ xv, int npts, int minRight,
                                                      int maxRight, double* __restrict__ Lout,
                                                      double* __restrict__ Tout, double* __restrict__ pv,
                                                      double* __restrict__ Pv)
{
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= numCells) return;
    const double n = dens[m];
    const size_t stride = static_cast<size_t>(numCells);

    double Labs = 0.;
    for (int ell = 0; ell < t.nrf; ++ell)
    {
        double op = n > 0. ? n * t.rfSigL[ell] : 0.;
        Labs += op * rf[ell * stride + m];
    }
    Lout[m] = Labs;

    const double factor = 1. / (4. * M_PI * t.vol[m]);
    double inputabs = 0.;
    for (int k = t.nrf - 1; k >= 0; --k)
    {
        double J = rf[k * stride + m] * factor / t.rfW[k];
        double term = t.rfSig[k] * (J + t.rfCmb[k]) * t.rfW[k];
        inputabs = (k == t.nrf - 1) ? term : inputabs + term;
    }
    double T = 0.;
    if (inputabs > 0.)
    {
        int i = locateNR(t.planck, t.nT, inputabs);
        if (i < 0)
            T = t.T[0];
        else if (i >= t.nT - 1)
            T = t.T[t.nT - 1];
        else
        {
            double x1 = t.planck[i], x2 = t.planck[i + 1], f1 = t.T[i], f2 = t.T[i + 1];
            T = f1 + ((inputabs - x1) / (x2 - x1)) * (f2 - f1);
        }
    }
    Tout[m] = n > 0. ? T : 0.;  // MediumSystem::indicativeDustTemperature: 0 without dust

    // the spectrum on the emission grid at index j: n * (sigma_em,j * B_T(lambda_j))
    auto ev = [&](int j) { return n * (t.emSig[j] * planckValue(T, t.emL[j])); };
    double* p = pv + static_cast<size_t>(m) * npts;
    double* P = Pv + static_cast<size_t>(m) * npts;
    const int nb = npts - 1;  // bins of the spectrum axis
    p[0] = minRight == 0 ? 0. : interpLogLog(xv[0], t.emL[minRight - 1], t.emL[minRight], ev(minRight - 1), ev(minRight));
    for (int i = 1; i < nb; ++i) p[i] = ev(minRight + i - 1);
    p[nb] = maxRight == t.nem ? 0. : interpLogLog(xv[nb], t.emL[maxRight - 1], t.emL[maxRight], ev(maxRight - 1), ev(maxRight));
    P[0] = 0.;
    for (int i = 0; i < nb; ++i)
    {
        double area = 0.;
        if (p[i] > 0 && p[i + 1] > 0)
        {
            double alpha = log(p[i + 1] / p[i]) / log(xv[i + 1] / xv[i]);
            area = p[i] * xv[i] * gln(-alpha, xv[i + 1] / xv[i]);
        }
        P[i + 1] = P[i] + area;
    }
    double norm = P[nb];
    if (norm > 0.)
        for (int i = 0; i <= nb; ++i)
        {
            p[i] /= norm;
            P[i] /= norm;
        }
}

// the leaf node of every octree cell (TreeSpatialGrid::nodeForCellIndex)
__global__ void cellNodeKernel(const int* __restrict__ tCell, int nodes, int* __restrict__ cellNode)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nodes) return;
    int c = tCell[n];
    if (c >= 0) cellNode[c] = n;
}

}  // namespace

cudaError_t launchDustCells(const DustEmissionDev& t, const double* dens, const double* rf, int numCells,
                            const double* xv, int npts, int minRight, int maxRight, double* L, double* T, double* pv,
                            double* Pv, cudaStream_t s)
{
    if (numCells <= 0) return cudaSuccess;
    dustCellKernel<<<(numCells + 255) / 256, 256, 0, s>>>(t, dens, rf, numCells, xv, npts, minRight, maxRight, L, T,
                                                          pv, Pv);
    return cudaGetLastError();
}

cudaError_t launchCellNodes(const int* tCell, int nodes, int* cellNode, cudaStream_t s)
{
    if (nodes <= 0) return cudaSuccess;
    cellNodeKernel<<<(nodes + 255) / 256, 256, 0, s>>>(tCell, nodes, cellNode);
    return cudaGetLastError();
}

}  // namespace skg
