/* SkgpuLifeCycle: the SKIRT-side bridge of the B200 photon-packet life cycle (include/skgpu.h).
 *
 * One class added to SKIRT/core. MonteCarloSimulation::runPrimaryEmission and
 * runSecondaryEmission (SKIRT/core/MonteCarloSimulation.cpp:172-245) call runPrimary / runSecondary,
 * runSecondaryEmissionIterations (:391-450) calls runSecondaryIteration, and
 * runMergedEmissionIterations runPrimaryIteration / runSecondaryIteration, in place of their
 * Parallel::call over performLifeCycle; when these return false (the bridge is
 * off, or the simulation uses something the library does not implement) SKIRT runs its own CPU
 * life cycle unchanged. Everything around the segment stays SKIRT's: ski parsing, setup, grid and
 * mesh construction, source normalisation and SourceSystem::prepareForLaunch, the instrument
 * flush, calibration and output, radiation-field communication, probes.
 *
 * The bridge is switched on per process by the command line's -g option (SkirtCommandLineHandler
 * calls setProcessEnabled(true) there, in place of GpuAcceleration::setProcessEnabled) or by the
 * environment variable SKGPU=1; a ski file then runs on the B200 with no change. SKGPU_DEVICE picks
 * the CUDA device (default: the process rank modulo the visible devices) and SKGPU_PRECISION=fp64
 * selects the reference-order FP64 walkers instead of the production precision.
 */
#ifndef SKGPULIFECYCLE_HPP
#define SKGPULIFECYCLE_HPP

#include <cstddef>
#include <string>

class MonteCarloSimulation;

class SkgpuLifeCycle final
{
public:
    /** Switches the bridge on or off for this process (the -g command-line option). */
    static void setProcessEnabled(bool enabled);

    /** True when the bridge is switched on (-g or SKGPU=1). */
    static bool isProcessEnabled();

    /** A one-line status for the simulation log: off, or the device and library in use. */
    static std::string status();

    /** Runs the primary-emission segment of Npp packets (this process's share of the history
        indices) on the B200 after SourceSystem::prepareForLaunch, adding the instrument tallies into
        the FluxRecorder arrays and the radiation field into MediumSystem's primary radiation field.
        Returns false, having done nothing, when the bridge is off or the simulation is not
        supported (the reason goes to the log); throws a FatalError when the library fails. */
    static bool runPrimary(MonteCarloSimulation* sim, size_t Npp);

    /** Runs the secondary (dust) emission segment of Npp packets from the primary radiation field
        in MediumSystem (after its communication between processes), adding the instrument tallies
        into the FluxRecorder arrays, secondary components included. Same return convention. */
    static bool runSecondary(MonteCarloSimulation* sim, size_t Npp);
    /** Runs one segment of Npp packets of the secondary emission iterations
        (MonteCarloSimulation::runSecondaryEmissionIterations): no detections, the segment's radiation
        field into MediumSystem's secondary field. Same return convention. */
    static bool runSecondaryIteration(MonteCarloSimulation* sim, size_t Npp);
    /** Runs the primary segment of Npp packets of a merged primary-secondary iteration
        (MonteCarloSimulation::runMergedEmissionIterations): no detections, the radiation field into
        MediumSystem's primary field. Same return convention. */
    static bool runPrimaryIteration(MonteCarloSimulation* sim, size_t Npp);

    /** Releases the device context (end of the process). */
    static void release();
};

#endif
