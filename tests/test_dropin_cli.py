"""The drop-in binary (the reference CLI with its CUDA backend translation
unit replaced by this library, mbs_fast_b200/host/Makefile `dropin`)
against the reference CLI on its CPU backend (oracle/_ref/mbs_po_ref, built
from the reference sources): same command line, same output files, results
within the FP64 tolerance."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "mbs_fast_b200", "_lib", "mbs_po_b200")
REFCLI = os.path.join(ROOT, "oracle", "_ref", "mbs_po_ref")
REFGPU = os.path.join(ROOT, "oracle", "_ref", "mbs_po_gpu_ref_fp64")

ARGS = ["--method", "po", "--particle", "1", "100", "40", "--refractive-index", "1.3116", "1e-9",
        "--wavelength-um", "0.532", "--max-reflections", "4", "--sobol", "64",
        "--scattering-grid", "0", "180", "48", "180", "--close"]


def _run(binary, backend, out, env_extra=None, extra_args=(), args=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    r = subprocess.run([binary] + (ARGS if args is None else args) + list(extra_args)
                       + ["--backend", backend, "--output", out],
                       capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    name = os.path.basename(out)
    rows = np.loadtxt(os.path.join(out, name + ".dat"), skiprows=1)
    with open(os.path.join(out, name + "_integrals.tsv")) as f:
        lines = [ln.rstrip("\n").split("\t") for ln in f if ln.strip()]
    integ = dict(zip(lines[0], lines[1]))
    return rows, integ, r.stdout + r.stderr


def _wl2(a, b):
    w = b[:, 1:2]                      # 2 pi dcos column
    return float(np.sqrt(np.sum(w * (a[:, 2:] - b[:, 2:]) ** 2) / np.sum(w * b[:, 2:] ** 2)))


@pytest.mark.gpu
@pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(REFCLI)),
                    reason="drop-in or reference CLI not built")
def test_dropin_matches_reference_cli(tmp_path):
    ref, ref_i, _ = _run(REFCLI, "cpu", str(tmp_path / "ref"))
    gpu, gpu_i, log = _run(DROPIN, "gpu", str(tmp_path / "gpu"), {"MBS_GPU_TIMING": "1"})
    assert "path=b200-fp64" in log          # the B200 library served the diffraction
    assert gpu.shape == ref.shape
    np.testing.assert_array_equal(gpu[:, :2], ref[:, :2])
    assert _wl2(gpu, ref) < 1e-7
    for k in ("Cext", "Csca"):
        assert abs(float(gpu_i[k]) / float(ref_i[k]) - 1) < 1e-7, k
    f32, f32_i, log32 = _run(DROPIN, "gpu", str(tmp_path / "f32"),
                             {"MBS_GPU_TIMING": "1", "MBS_B200_PRECISION": "fp32c"})
    assert "path=b200-fp32c" in log32
    assert _wl2(f32, ref) < 2e-5


@pytest.mark.gpu
@pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(REFGPU)),
                    reason="drop-in or the reference's CUDA build not built")
def test_dropin_matches_reference_cuda_build(tmp_path):
    """Direct mode (no --fft): the reference's own CUDA FP64 build and the
    drop-in on the same command line and device, .dat rows and integrals."""
    ref, ref_i, ref_log = _run(REFGPU, "gpu", str(tmp_path / "ref"))
    assert "Phase 2 (diffraction, CUDA)" in ref_log
    gpu, gpu_i, log = _run(DROPIN, "gpu", str(tmp_path / "gpu"), {"MBS_GPU_TIMING": "1"})
    assert "path=b200-fp64" in log
    assert gpu.shape == ref.shape
    np.testing.assert_array_equal(gpu[:, :2], ref[:, :2])
    assert _wl2(gpu, ref) < 1e-7
    for k in ("Cext", "Csca"):
        assert abs(float(gpu_i[k]) / float(ref_i[k]) - 1) < 1e-7, k


@pytest.mark.gpu
@pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(REFGPU)),
                    reason="drop-in or the reference's CUDA build not built")
def test_dropin_fft_phi_matches_reference_cuda_build(tmp_path):
    """--fft: the reference's CUDA build (its own FFT-phi path, cuFFT) and the
    drop-in (direct evaluation on the reduced azimuth grid and the device
    interpolation of this library) on the same command line; both FP64."""
    ref, ref_i, ref_log = _run(REFGPU, "gpu", str(tmp_path / "ref"), extra_args=["--fft"])
    assert "FFT angular interpolation" in ref_log
    gpu, gpu_i, log = _run(DROPIN, "gpu", str(tmp_path / "gpu"), {"MBS_GPU_TIMING": "1"},
                           extra_args=["--fft"])
    assert "path=b200-fp64" in log and "nPhiOut=48" in log
    assert gpu.shape == ref.shape
    np.testing.assert_array_equal(gpu[:, :2], ref[:, :2])
    assert _wl2(gpu, ref) < 1e-7
    for k in ("Cext", "Csca"):
        assert abs(float(gpu_i[k]) / float(ref_i[k]) - 1) < 1e-7, k


@pytest.mark.gpu
@pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(REFGPU)),
                    reason="drop-in or the reference's CUDA build not built")
def test_dropin_eps1_and_beam_stats_knobs(tmp_path):
    """MBS_GPU_EPS1 moves the singular-edge threshold in both builds alike
    (the drop-in equals the reference's CUDA FP64 build under the same
    override), and MBS_GPU_BEAM_STATS=1 prints per-batch beam statistics
    whose beam totals agree with the reference build's."""
    import re
    env = {"MBS_GPU_EPS1": "1e-4", "MBS_GPU_BEAM_STATS": "1"}
    ack = ["--allow-experimental-environment"]   # the CLI's guard for result-affecting knobs
    ref, ref_i, ref_log = _run(REFGPU, "gpu", str(tmp_path / "ref"), env, extra_args=ack)
    gpu, gpu_i, log = _run(DROPIN, "gpu", str(tmp_path / "gpu"), dict(env, MBS_GPU_TIMING="1"),
                           extra_args=ack)
    assert "path=b200-fp64" in log
    assert _wl2(gpu, ref) < 1e-7
    for k in ("Cext", "Csca"):
        assert abs(float(gpu_i[k]) / float(ref_i[k]) - 1) < 1e-7, k

    def beams(text):
        return sum(int(m) for m in re.findall(r"GPU beam stats orient=\d+ beams=(\d+)", text))
    assert beams(log) > 0 and beams(log) == beams(ref_log)


@pytest.mark.gpu
@pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(REFCLI)),
                    reason="drop-in or reference CLI not built")
def test_dropin_variable_phi_so3_matches_reference_cli(tmp_path):
    """--so3-quaternion: the reference driver's variable-phi averaging, which
    diffracts each prepared chunk on several theta-row groups with their own
    azimuth counts (new grids call after call, TracerPOTotal.cpp:6057-6830);
    the drop-in's result equals the reference CLI's CPU result."""
    args = [a for a in ARGS]
    i = args.index("--sobol")
    args[i:i + 2] = ["--so3-quaternion", "32"]
    ref, ref_i, _ = _run(REFCLI, "cpu", str(tmp_path / "ref"), args=args)
    gpu, gpu_i, log = _run(DROPIN, "gpu", str(tmp_path / "gpu"), {"MBS_GPU_TIMING": "1"}, args=args)
    assert "path=b200-fp64" in log
    assert gpu.shape == ref.shape
    np.testing.assert_array_equal(gpu[:, :2], ref[:, :2])
    assert _wl2(gpu, ref) < 1e-7
    for k in ("Cext", "Csca"):
        assert abs(float(gpu_i[k]) / float(ref_i[k]) - 1) < 1e-7, k


CACHE_CHECK = os.path.join(ROOT, "mbs_fast_b200", "_lib", "mbs_dropin_cache_check")


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(CACHE_CHECK), reason="cache check not built")
def test_dropin_packed_beam_cache():
    """HandleOrientationsToLocalGpuOnDevice with a cache token (the
    reference's multi-GPU theta-group path, which a one-GPU CLI run never
    takes): tests/dropin_cache_check.cpp traces a column with the reference,
    then fills and hits the cache on two grids and refills it for another
    range; every result equals the uncached call bit for bit."""
    env = dict(os.environ, MBS_GPU_TIMING="1")
    r = subprocess.run([CACHE_CHECK], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    assert r.stdout.strip().endswith("OK")
    assert r.stderr.count("cache=fill") == 2 and r.stderr.count("cache=hit") == 3, r.stderr[-3000:]


@pytest.mark.gpu
@pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(REFCLI)),
                    reason="drop-in or reference CLI not built")
def test_dropin_noshadow_output_matches_reference_cli(tmp_path):
    """--no-shadow-output (HandlerPO::ComputeNoShadow, the kernels that also
    accumulate the sums over internal beams): the full and the no-shadow .dat
    rows and integrals of the drop-in against the reference CLI, FP64 and
    FP32C."""
    def run(binary, backend, out, env=None):
        rows, integ, log = _run(binary, backend, out, env, ["--no-shadow-output"])
        name = os.path.basename(out)
        ns = np.loadtxt(os.path.join(out, name + "_noshadow.dat"), skiprows=1)
        with open(os.path.join(out, name + "_noshadow_integrals.tsv")) as f:
            lines = [ln.rstrip("\n").split("\t") for ln in f if ln.strip()]
        return rows, integ, ns, dict(zip(lines[0], lines[1])), log

    ref, ref_i, ref_ns, ref_nsi, _ = run(REFCLI, "cpu", str(tmp_path / "ref"))
    for prec, gate in (("fp64", 1e-7), ("fp32c", 1e-4)):
        gpu, gpu_i, ns, nsi, log = run(DROPIN, "gpu", str(tmp_path / prec),
                                       {"MBS_GPU_TIMING": "1", "MBS_B200_PRECISION": prec})
        assert "path=b200-" + prec in log
        assert gpu.shape == ref.shape and ns.shape == ref_ns.shape
        np.testing.assert_array_equal(ns[:, :2], ref_ns[:, :2])
        assert _wl2(gpu, ref) < gate, prec
        assert _wl2(ns, ref_ns) < gate, prec
        if prec == "fp64":
            for k in ("Csca",):
                assert abs(float(nsi[k]) / float(ref_nsi[k]) - 1) < 1e-7, k
