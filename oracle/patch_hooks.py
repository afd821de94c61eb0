"""Build step of the bridged reference program (oracle/ref.mk target `bridge`): copies the two
reference source files that host the life-cycle hooks into oracle/_ref/patched/ and inserts the hooks
there (the reference tree itself is never modified):

- SKIRT/core/MonteCarloSimulation.cpp: runPrimaryEmission and runSecondaryEmission hand their
  segment to SkgpuLifeCycle::runPrimary / runSecondary, each segment of
  runSecondaryEmissionIterations to SkgpuLifeCycle::runSecondaryIteration, and the primary and
  secondary segments of runMergedEmissionIterations to runPrimaryIteration / runSecondaryIteration,
  keeping the
  Parallel::call over performLifeCycle as the path taken when the bridge declines;
- SKIRT/main/SkirtCommandLineHandler.cpp: the -g option switches the bridge on (in place of the
  reference's runtime-loaded GPU layer) and the log reports the bridge's status.

    python3 oracle/patch_hooks.py <reference root> <output directory>

Every replacement must match exactly once; otherwise the script stops with an error.
"""
import os
import re
import sys


def patch(text, pattern, repl, what):
    new, n = re.subn(pattern, repl, text, flags=re.S)
    if n != 1:
        raise SystemExit(f"patch_hooks: {what}: expected one match, found {n}")
    return new


def main():
    ref, out = sys.argv[1], sys.argv[2]
    os.makedirs(out, exist_ok=True)

    src = open(os.path.join(ref, "SKIRT", "core", "MonteCarloSimulation.cpp")).read()
    src = patch(src, r'(#include "MonteCarloSimulation\.hpp"\n)', r'\1#include "SkgpuLifeCycle.hpp"\n', "include")
    src = patch(src,
                r'(\n[ \t]*auto parallel = find<ParallelFactory>\(\)->parallelDistributed\(lifeCycleThreadLimit\(_config\)\);'
                r'\s*parallel->call\(\s*Npp, \[this\]\(size_t i, size_t n\) \{ performLifeCycle\(i, n, true, true, '
                r'_config->hasRadiationField\(\)\); \}\);)',
                r'\n        if (!SkgpuLifeCycle::runPrimary(this, Npp))\n        {\1\n        }',
                "primary segment")
    src = patch(src,
                r'(\n[ \t]*auto parallel = find<ParallelFactory>\(\)->parallelDistributed\(lifeCycleThreadLimit\(_config\)\);'
                r'\s*parallel->call\(Npp, \[this, storeRF\]\(size_t i, size_t n\) \{ performLifeCycle\(i, n, false, true, '
                r'storeRF\); \}\);)',
                r'\n        if (!SkgpuLifeCycle::runSecondary(this, Npp))\n        {\1\n        }',
                "secondary segment")
    src = patch(src,
                r'(\n[ \t]*parallel->call\(Npp, \[this\]\(size_t i, size_t n\) \{ performLifeCycle\(i, n, false, false, true\); \}\);)',
                r'\n            if (!SkgpuLifeCycle::runSecondaryIteration(this, Npp))\n            {\1\n            }',
                "secondary iteration segment")
    src = patch(src,
                r'(\n[ \t]*parallel->call\(Npp1, \[this\]\(size_t i, size_t n\) \{ performLifeCycle\(i, n, true, false, true\); \}\);)',
                r'\n            if (!SkgpuLifeCycle::runPrimaryIteration(this, Npp1))\n            {\1\n            }',
                "merged primary iteration segment")
    src = patch(src,
                r'(\n[ \t]*parallel->call\(Npp2, \[this\]\(size_t i, size_t n\) \{ performLifeCycle\(i, n, false, false, true\); \}\);)',
                r'\n            if (!SkgpuLifeCycle::runSecondaryIteration(this, Npp2))\n            {\1\n            }',
                "merged secondary iteration segment")
    with open(os.path.join(out, "MonteCarloSimulation.cpp"), "w") as f:
        f.write(src)

    src = open(os.path.join(ref, "SKIRT", "main", "SkirtCommandLineHandler.cpp")).read()
    src = patch(src, r'(#include "GpuAcceleration\.hpp"\n)', r'\1#include "SkgpuLifeCycle.hpp"\n', "include")
    src = patch(src, r'if \(_args\.isPresent\("-g"\)\) GpuAcceleration::setProcessEnabled\(true\);',
                'if (_args.isPresent("-g")) SkgpuLifeCycle::setProcessEnabled(true);', "-g option")
    src = patch(src, r'log->info\("GPU acceleration is " \+ GpuAcceleration::status\(\)\);',
                'log->info("GPU acceleration is " + SkgpuLifeCycle::status());', "status line")
    with open(os.path.join(out, "SkirtCommandLineHandler.cpp"), "w") as f:
        f.write(src)


if __name__ == "__main__":
    main()
