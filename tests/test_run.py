"""time_advance with its monitor and output (ns3d_run, maincycle.cpp:7-112),
the segmented loop under it (ns3d_time_advance_segment) and the file writers
it uses: the spectrum file and the statistics table of isotropic_post_process.

CPU: the writers reproduce the reference's files byte for byte. GPU: the
segmented loop repeats ns3d_time_advance bit for bit; ns3d_run writes the same
files as the reference's own time_advance, with the same values to the digits
printed."""
import ctypes
import os
import re
import tempfile

import numpy as np
import pytest

import ns3d_cpp_b200 as ns
from ns3d_cpp_b200 import _lib, initial
from ns3d_cpp_b200.solver import TurbStats
from conftest import ref_cfg

needs_ref = pytest.mark.skipif(
    not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                    "libns3d_ref.so")),
    reason="reference build (oracle/_ref) not present")

STATS_NAMES = ["kinetic_energy", "tke", "u_rms", "dissipation", "taylor", "eta", "u_eta",
               "tau_eta", "taylor_li", "re_lambda", "mach_t"]


def params_for(cfg):
    with tempfile.NamedTemporaryFile("w", suffix=".in", delete=False) as f:
        f.write("".join(f"{k} = {v}\n" for k, v in cfg.items()))
        path = f.name
    try:
        return ns.read_solver_params_from_file(path)
    finally:
        os.unlink(path)


def tgv(n, seed=3):
    return np.ascontiguousarray(initial.taylor_green(n, Ma=0.3, perturb=0.05, seed=seed))


def dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def read_bytes(path):
    with open(path, "rb") as f:
        return f.read()


@needs_ref
def test_spectrum_and_stats_writers_match_reference_files(oracle_mod):
    n = 16
    cfg = ref_cfg(n, Ma=0.3)
    r = oracle_mod.Ref(cfg)
    r.set_primitive(tgv(n))
    lib = _lib.load()
    with tempfile.TemporaryDirectory() as d:
        r.isotropic_post(d, 0.125)
        r.isotropic_post(d, 0.25)
        spec = os.path.join(d, "output", "output_time_0.12500_spectrum.dat")
        ref_spec = read_bytes(spec)
        Ek = np.array([float(line.split()[1]) for line in ref_spec.decode().splitlines()])
        assert len(Ek) == 2 * n + 1
        ours = os.path.join(d, "spec.dat")
        assert lib.ns3d_spectrum_write(ours.encode(), dp(Ek), len(Ek)) == 0
        assert read_bytes(ours) == ref_spec
        # the statistics table: header once, then one row per call
        ref_stats = read_bytes(os.path.join(d, "output", "turbulence_stats.dat"))
        rows = ref_stats.decode().splitlines()
        assert len(rows) == 3
        ours = os.path.join(d, "stats.dat")
        for row in rows[1:]:
            v = [float(x) for x in row.split()]
            s = TurbStats()
            for name, x in zip(STATS_NAMES, v[1:]):
                setattr(s, name, x)
            assert lib.ns3d_stats_write(ours.encode(), v[0], ctypes.byref(s)) == 0
        assert read_bytes(ours) == ref_stats
        assert lib.ns3d_spectrum_write(os.path.join(d, "no", "x.dat").encode(), dp(Ek), 3) == 5
        assert lib.ns3d_spectrum_write(ours.encode(), dp(Ek), 0) == 1


def run_cfg(n, **kw):
    c = ref_cfg(n, Ma=0.3, Post_BasicField="True", IsotropicAnalyse="True", monitor_Res="True",
                monitor_Energy="True", monitor_Stepfreq=2, max_steps=9, TotalTime=10.0,
                output_Timefreq=0.1)
    c.update(kw)
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32acc64"])
def test_segments_repeat_time_advance(precision):
    """Segments that end after every output step, continued to max steps, give
    the same states, clock and dt as one time_advance call."""
    p = params_for(run_cfg(16, TotalTime=0.5))
    p.precision = ns.solver.PRECISION[precision]
    with ns.Solver(p) as a, ns.Solver(p) as b:
        a.upload_primitive(tgv(16))
        b.upload_primitive(tgv(16))
        ta, ka = a.time_advance(40)
        steps, outputs, t, ended = 0, 0, 0.0, False
        while steps < 40 and not ended:
            t, k, ev = b.time_advance_segment(40 - steps)
            steps += k
            outputs += "output" in ev
            ended = "end" in ev
            if k == 0:
                break
        assert ended and (t, steps) == (ta, ka) and abs(ta - 0.5) < 1e-12
        # the output times 0.1 .. 0.4 at least (0.5 coincides with TotalTime)
        assert outputs >= 4
        assert np.array_equal(a.download_primitive(with_T_c=True), b.download_primitive(with_T_c=True))
        assert a.last_dt() == b.last_dt()


def read_table(path, skip):
    with open(path) as f:
        rows = f.read().splitlines()[skip:]
    return np.array([[float(x) for x in r.split()] for r in rows])


def tree(root):
    out = []
    for dirpath, _, files in os.walk(root):
        out += [os.path.relpath(os.path.join(dirpath, f), root) for f in files]
    return sorted(out)


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(), dict(TotalTime=0.3, monitor_Stepfreq=3, max_steps=20)],
                         ids=["max_steps", "total_time"])
def test_run_writes_the_reference_files(oracle_mod, kw):
    n = 16
    cfg = run_cfg(n, **kw)
    W = tgv(n, seed=5)
    r = oracle_mod.Ref(cfg)
    r.set_primitive(W)
    with tempfile.TemporaryDirectory() as d:
        dr, dg = os.path.join(d, "ref"), os.path.join(d, "gpu")
        os.makedirs(dr)
        r.time_advance(dr)
        with ns.Solver(params_for(cfg)) as s:
            s.upload_primitive(W)
            t, k = s.run(dg, verbose=False)
        files = tree(os.path.join(dr, "output"))
        assert files == tree(os.path.join(dg, "output"))
        assert "output_residuals.dat" in files and "turbulence_stats.dat" in files
        assert any(f.startswith("time_") for f in files)
        for f in files:
            a, b = os.path.join(dr, "output", f), os.path.join(dg, "output", f)
            if f == "output_residuals.dat":
                A, B = read_table(a, 2), read_table(b, 2)
                assert np.array_equal(A[:, 0], B[:, 0])
                assert np.allclose(B, A, rtol=1e-6, atol=0)
            elif f == "turbulence_stats.dat":
                assert read_bytes(a).splitlines()[0] == read_bytes(b).splitlines()[0]
                A, B = read_table(a, 1), read_table(b, 1)
                assert np.array_equal(A[:, 0], B[:, 0])
                assert np.allclose(B, A, rtol=1e-5, atol=0)
            elif f.endswith("_spectrum.dat"):
                A, B = read_table(a, 0), read_table(b, 0)
                assert np.array_equal(A[:, 0], B[:, 0])
                assert np.all(np.abs(B[:, 1] - A[:, 1]) <= 2e-5 * np.abs(A[:, 1])
                              + 1e-12 * np.max(np.abs(A[:, 1])))
            else:
                A, B = read_table(a, 3), read_table(b, 3)
                assert read_bytes(a).splitlines()[:3] == read_bytes(b).splitlines()[:3]
                assert np.allclose(B, A, rtol=1e-7, atol=1e-12)
    if "TotalTime" in kw:
        assert abs(t - 0.3) < 1e-12 and k < 20
    else:
        assert k == 9


def _stdout_lines(text):
    """The "Completed step" and "[Step" lines, wall-clock fields removed."""
    out = []
    for line in text.splitlines():
        if line.startswith("Completed step"):
            out.append(line)
        elif line.startswith("[Step"):
            out.append(re.sub(r"Time/step=\S+s  Elapsed=\S+s", "", line))
    return out


@needs_ref
@pytest.mark.gpu
def test_run_prints_the_reference_step_lines(oracle_mod, capfd):
    """ns3d_run's stdout against the reference's own time_advance
    (maincycle.cpp:56-86): one "Completed step" line per step with the same
    step numbers and times, the monitor lines in the same places, the same
    number formats (the stream turns to fixed 6 decimals at the first monitor
    line). The first line's time is compared by value: an earlier reference
    run in this process may have left its stream in fixed format."""
    n = 16
    cfg = run_cfg(n, TotalTime=0.3, monitor_Stepfreq=3, max_steps=20)
    W = tgv(n, seed=5)
    libc = ctypes.CDLL(None)
    r = oracle_mod.Ref(cfg)
    r.set_primitive(W)
    with tempfile.TemporaryDirectory() as d:
        dr, dg = os.path.join(d, "ref"), os.path.join(d, "gpu")
        os.makedirs(dr)
        libc.fflush(None)
        capfd.readouterr()
        r.time_advance(dr)
        libc.fflush(None)
        ref_out = capfd.readouterr().out
        with ns.Solver(params_for(cfg)) as s:
            s.upload_primitive(W)
            t, k = s.run(dg, verbose=True)
            times = s.step_times()
        libc.fflush(None)
        gpu_out = capfd.readouterr().out
    a, b = _stdout_lines(ref_out), _stdout_lines(gpu_out)
    assert sum(x.startswith("Completed") for x in a) == k > 3
    assert len(a) == len(b)
    head_a, head_b = a[0].split("Time = "), b[0].split("Time = ")
    assert head_a[0] == head_b[0]
    ta, tb = float(head_a[1].split(" / ")[0]), float(head_b[1].split(" / ")[0])
    assert abs(ta - tb) <= 5e-7 * max(1.0, abs(tb))  # 6 decimals or 6 digits
    assert a[1:] == b[1:]
    assert "Simulation complete. Total time: " in gpu_out
    # the record of the last segment ends at the returned time
    assert len(times) >= 1 and times[-1] == t


@pytest.mark.gpu
def test_run_argument_errors():
    p = params_for(run_cfg(16))
    with ns.Solver(p) as s, tempfile.TemporaryDirectory() as d:
        s.upload_primitive(tgv(16))
        with pytest.raises(ns.NS3DError) as e:
            s.run(d, max_steps=-1)
        assert e.value.status == 1
    p = params_for(run_cfg(16, monitor_Stepfreq=0))
    with ns.Solver(p) as s, tempfile.TemporaryDirectory() as d:
        s.upload_primitive(tgv(16))
        with pytest.raises(ns.NS3DError) as e:
            s.run(d)
        assert e.value.status == 1
