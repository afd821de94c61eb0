"""Explicit absorption (PhotonPacketOptions::explicitAbsorption) on the GPU: the FP64 life cycle
equals the oracle history by history (forced and free propagation, with the radiation field and
the panchromatic galaxy's tabulated cross sections), the production FP32 walkers stay within noise
of it, and the images agree with the reference's own explicit-absorption runs (z-scores)."""
import numpy as np
import pytest

from helpers import zscores
from skgpu import Scene, abi, workloads
from test_gpu_parity import assert_close_runs, run_both

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("forced", [True, False])
def test_gpu_explicit_absorption_matches_oracle(golden, gpu_backend, oracle_backend, forced):
    sc = Scene.from_export(golden("shell_c16.npz"))
    sc.explicit_absorption = True
    sc.force_scattering = forced
    if forced:
        sc.store_rf = True
        sc.rf = dict(num_bins=1, borders=np.array([0.5e-6, 0.6e-6]), ellv=np.array([-1, 0, -1], np.int32))
    rg, ro = run_both(sc, gpu_backend, oracle_backend, 20000, seed=13)
    assert_close_runs(rg, ro)
    if forced:
        assert rg.rf.sum() == pytest.approx(ro.rf.sum(), rel=1e-6)
        assert np.mean(np.isclose(rg.rf, ro.rf, rtol=1e-9, atol=0)) > 0.99


def test_gpu_explicit_absorption_galaxy_matches_oracle(gpu_backend, oracle_backend):
    sc = workloads.galaxy_octree(npix=32, nlambda=20, max_level=5, max_dust_fraction=1e-4)
    sc.explicit_absorption = True
    rg, ro = run_both(sc, gpu_backend, oracle_backend, 4000, seed=8)
    assert_close_runs(rg, ro)
    assert rg.rf.sum() == pytest.approx(ro.rf.sum(), rel=1e-6)


@pytest.mark.parametrize("forced", [True, False])
def test_gpu_explicit_absorption_matches_reference_statistics(golden, gpu_backend, forced):
    z = golden("shell_c16.npz")
    e = golden("shell_c16_explicit.npz")
    tag = "forced" if forced else "free"
    sc = Scene.from_export(z)
    sc.explicit_absorption = True
    sc.force_scattering = forced
    sc.upload(gpu_backend)
    n = int(e["ref_npp"])
    for precision in (abi.PREC_FP64_EXACT, abi.PREC_FP32):
        res = sc.run(gpu_backend, n, seed=17, precision=precision)
        st = res[0]["stats"][:, 0]
        ref = e[f"ref_{tag}_frame_w"]
        zs = zscores(st[1], st[2], n, ref[1], ref[2], n)
        assert abs(zs.mean()) < 0.1 and 0.85 < zs.std() < 1.15
        sst = res[1]["stats"][:, 0]
        rs = e[f"ref_{tag}_sedstats"]
        assert abs(zscores(sst[1:2], sst[2:3], n, rs[1:2], rs[2:3], n)[0]) < 4
