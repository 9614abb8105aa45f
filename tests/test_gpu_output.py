"""GPU checks of the device-path output (reference text formats, async
writers, exact checkpoints).

* sclbm_domain_write_text writes, synchronously or from a worker thread, the
  same bytes as the host writer (itself pinned byte for byte to the compiled
  reference in test_output_cpu.py) applied to the downloaded fields;
* Fluid::restart_from_file's layout reads the nine population files back;
* a checkpoint reloaded into a domain continues the run bit for bit in every
  storage precision, and is refused by a domain of another shape.
"""
import numpy as np
import pytest

import cases
import gpu_runner

pytestmark = pytest.mark.gpu

RUNS = cases.all_cases()
PRECS = ["FP64", "FP32_SHIFTED", "FP16_SHIFTED"]


def _domain(sclbm, prec, name="porous_96x48", steps=5):
    d = gpu_runner.make_domain(sclbm, RUNS[name], getattr(sclbm, prec), rho_ref=(0.5, 1.5))
    d.step(steps)
    return d


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("asynchronous", [False, True])
def test_write_text_matches_host_writer(sclbm, tmp_path, prec, asynchronous):
    d = _domain(sclbm, prec)
    nx, ny, N = d.nx, d.ny, d.N
    for comp in (0, 1):
        d.write_density(comp, tmp_path / f"rho{comp}.txt", asynchronous)
        d.save_state(comp, tmp_path / f"s_rho{comp}", tmp_path / f"s_ux{comp}",
                     tmp_path / f"s_uy{comp}", 7, asynchronous)
        d.write_f(comp, tmp_path / f"f{comp}", asynchronous)
    # later steps queued behind the asynchronous copies must not leak into them
    snapshot = [(d.download_rho(c), d.download_velocity(c), d.download_f(c)) for c in (0, 1)]
    d.step(3)
    sclbm.io_wait()
    for comp, (rho, (ux, uy), f) in enumerate(snapshot):
        for path, v in ((f"rho{comp}.txt", rho), (f"s_rho{comp}_7.txt", rho),
                        (f"s_ux{comp}_7.txt", ux), (f"s_uy{comp}_7.txt", uy)):
            ref = tmp_path / ("ref_" + path)
            sclbm.write_rows(ref, v, nx, ny)
            assert (tmp_path / path).read_bytes() == ref.read_bytes(), (prec, path)
        for i in range(9):
            ref = tmp_path / f"ref_f{comp}_{i}.txt"
            sclbm.write_rows(ref, f[i * N:(i + 1) * N], nx, ny)
            assert (tmp_path / f"f{comp}_{i}.txt").read_bytes() == ref.read_bytes(), (prec, i)


def test_async_write_failure_is_reported(sclbm, tmp_path):
    d = _domain(sclbm, "FP32_SHIFTED")
    d.write_density(0, tmp_path / "missing_dir" / "rho.txt", asynchronous=True)
    with pytest.raises(RuntimeError):
        sclbm.io_wait()
    sclbm.io_wait()  # the failure was reported once


@pytest.mark.parametrize("prec", PRECS)
def test_restart_from_text_files(sclbm, tmp_path, prec):
    d = _domain(sclbm, prec)
    d.write_f(1, tmp_path / "f")
    e = gpu_runner.make_domain(sclbm, RUNS["porous_96x48"], getattr(sclbm, prec), rho_ref=(0.5, 1.5))
    e.restart_from_file(0, tmp_path / "f")
    want = np.concatenate([sclbm.read_rows(tmp_path / f"f_{i}.txt", d.nx, d.ny) for i in range(9)])
    got = e.download_f(0)
    if prec == "FP64":
        assert np.array_equal(got, want)
    else:
        # stored again in the shifted form: within its rounding
        tol = 1e-6 if prec == "FP32_SHIFTED" else 2e-3
        assert np.max(np.abs(got - want)) <= tol


@pytest.mark.parametrize("prec", PRECS)
def test_checkpoint_continues_bit_for_bit(sclbm, tmp_path, prec):
    d = _domain(sclbm, prec, steps=11)
    ck = tmp_path / "run.ck"
    d.checkpoint_save(ck)
    d.step(9)
    a = [d.download_f(c) for c in (0, 1)]
    e = gpu_runner.make_domain(sclbm, RUNS["porous_96x48"], getattr(sclbm, prec), rho_ref=(0.5, 1.5))
    e.checkpoint_load(ck)
    e.step(9)
    for c in (0, 1):
        assert e.download_f(c).tobytes() == a[c].tobytes()


def test_checkpoint_refuses_other_domains(sclbm, tmp_path):
    d = _domain(sclbm, "FP32_SHIFTED")
    ck = tmp_path / "run.ck"
    d.checkpoint_save(ck)
    other = gpu_runner.make_domain(sclbm, RUNS["porous_96x48"], sclbm.FP64)
    with pytest.raises(ValueError):
        other.checkpoint_load(ck)
    other = gpu_runner.make_domain(sclbm, RUNS["channel_80x32"], sclbm.FP32_SHIFTED)
    with pytest.raises(ValueError):
        other.checkpoint_load(ck)
    with pytest.raises(ValueError):
        d.checkpoint_load(__file__)  # not a checkpoint
    with pytest.raises(RuntimeError):
        d.checkpoint_load(tmp_path / "missing.ck")
