"""Run-control front end on the GPU: the lbmc_run program and lbmc_run()
against the engine driven step by step, the reference's steady-state rule
(LBM-C/index.cu:102-142), the non-finite exit, and checkpoint/restart."""
import json
import os
import subprocess

import numpy as np
import pytest

from cases import make_case

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "lbm-c_b200", "lbmc_run")


def channel(tmp_path, lx=128, ly=64, g=1e-6, extra="", **fields):
    """Poiseuille channel: D2Q9 BGK, tau 0.8, Guo force g along x, bounceback
    rows at y = 0 and y = Ly - 1; domain files + input file."""
    dom = tmp_path / "dom"
    dom.mkdir(exist_ok=True)
    n = lx * ly
    y = np.arange(n) // lx
    por = np.zeros(n)
    por[(y == 0) | (y == ly - 1)] = 1.0
    np.save(dom / "Porosity.npy", por.reshape(ly, lx))
    np.save(dom / "ForceX.npy", np.full(n, g))
    np.save(dom / "ForceY.npy", np.zeros(n))
    for k, v in fields.items():
        np.save(dom / f"{k}.npy", v)
    text = (f"ProjName channel\nDomainFile {dom}\nOutputFile {tmp_path / 'out'}\nTau 0.8\n"
            f"Lx {lx}\nLy {ly}\nColType BGK\nForce 1\nMicroBC 0\nMacroBC 0\nOutputVars 1 1 0 1 0\n"
            f"ScreenNode {lx // 2} {ly // 2} 0\n" + extra)
    p = tmp_path / "input.txt"
    p.write_text(text)
    return str(p), dict(geometry=por, force=np.stack([np.full(n, g), np.zeros(n)]))


def engine(lbmc, lx, ly, arrays, **kw):
    cfg = lbmc.make_config("d2q9", (lx, ly, 1), tau=0.8, collision_type=lbmc.BGK, forcing=True, **kw)
    dom, keep = lbmc.make_domain(lx * ly, 2, 9, arrays["geometry"], arrays["force"])
    eng = lbmc.Engine(cfg, dom)
    eng._keep = keep
    return eng


def load_solution(out, step):
    idx = json.loads((out / "index.json").read_text())
    for s in idx["Base"]["Zone"]["FlowSolutions"]:
        if s["name"] == f"Solution @ Time = {step}":
            return {k: np.load(out / v).reshape(-1) for k, v in s["fields"].items()}
    raise KeyError(step)


def test_cli_channel_matches_engine(lbmc, tmp_path):
    path, arrays = channel(tmp_path, extra="MaxT 400\nFileOut 200\nScreenMes 100\nSteadyCheck 0\n")
    r = subprocess.run([CLI, path, "--quiet"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    with engine(lbmc, 128, 64, arrays) as eng:
        for step in (200, 400):
            eng.iterate(200, lbmc.STORE_MACROS | lbmc.SYNC)
            sol = load_solution(tmp_path / "out", step)
            np.testing.assert_array_equal(sol["VelocityX"], eng.u()[0])
            np.testing.assert_array_equal(sol["VelocityY"], eng.u()[1])
            np.testing.assert_array_equal(sol["Density"], eng.rho())
    # Screen report (not quiet): the reference's line format.
    r = subprocess.run([CLI, path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "time = 100; rho = " in r.stdout and "resid = " in r.stdout


def test_steady_state_stop_follows_the_reference_rule(lbmc, tmp_path):
    check, tol = 500, 1e-6
    path, arrays = channel(tmp_path, lx=32, ly=24, extra=f"MaxT 200000\nFileOut 0\nSteadyCheck {check}\n"
                                                          f"Tolerance {tol}\n")
    st, res = lbmc.run(path)
    assert st == lbmc.OK and res.steady == 1 and res.steps < 200000
    assert max(res.residual) < tol
    # The same rule evaluated here from the engine's FP64 kinetic energy:
    # r(t) = |KE(t) - KE(t - C)| / C / KE(t) into a ring of three (starting
    # at 1), stop at the first check where all three are below Tolerance.
    ring, prev, t = [1.0, 1.0, 1.0], 0.0, 0
    with engine(lbmc, 32, 24, arrays) as eng:
        while True:
            eng.iterate(check, lbmc.REDUCE_DIAG | lbmc.STORE_MACROS | lbmc.SYNC)
            t += check
            ke = eng.diag().kinetic_energy
            ring[t % 3] = abs(ke - prev) / check / ke
            prev = ke
            if all(r < tol for r in ring):
                break
        u_stop = eng.u()[0]
    assert res.steps == t
    sol = load_solution(tmp_path / "out", t)  # the stop writes a solution
    np.testing.assert_array_equal(sol["VelocityX"], u_stop)


def test_nonfinite_run_exits_with_1(lbmc, tmp_path):
    """A NaN planted on the host in the initial populations (Init 2): the
    first steady-state check sees a non-finite state, the run writes a
    solution and lbmc_run exits with 1, as the reference does
    (LBM-C/index.cu:130-133)."""
    n = 32 * 24
    w = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
    f0 = np.repeat(w[:, None], n, axis=1)
    f0[3, 400] = np.nan
    path, _ = channel(tmp_path, lx=32, ly=24, extra="Init 2\nMaxT 5000\nFileOut 0\nSteadyCheck 10\n"
                                                    "Tolerance 1e-12\n", Populations=f0)
    r = subprocess.run([CLI, path, "--quiet"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 1, (r.returncode, r.stderr)
    st, res = lbmc.run(path)
    assert st == lbmc.ERR_NAN and res.nonfinite == 1 and res.steps == 10
    idx = json.loads((tmp_path / "out" / "index.json").read_text())
    assert idx["Base"]["BaseIterativeData"]["IterationValues"][-1] == 10


@pytest.mark.parametrize("streaming", ["shift", "aa"])
def test_checkpoint_restart_is_exact(lbmc, tmp_path, streaming):
    """Populations fetched at an odd step and given back as the initial
    state (LBMC_INIT_F) continue exactly as an uninterrupted run."""
    sm = lbmc.STREAM_AA if streaming == "aa" else lbmc.STREAM_SHIFT
    case = make_case("d3q15", (19, 11, 9), 3, True, solids=0.08, partial=0.15, micro="zh",
                     macro="random", seed=9)
    with lbmc.Engine.from_case(case, streaming=sm) as eng:
        eng.iterate(137, lbmc.SYNC)
        f_mid = eng.f()
        eng.iterate(100, lbmc.STORE_MACROS | lbmc.SYNC)
        f_end, u_end = eng.f(), eng.u()
    case.f0 = f_mid
    with lbmc.Engine.from_case(case, storage=lbmc.F32, init_type=lbmc.INIT_F, streaming=sm) as eng:
        eng.iterate(100, lbmc.STORE_MACROS | lbmc.SYNC)
        np.testing.assert_array_equal(eng.f(), f_end)
        np.testing.assert_array_equal(eng.u(), u_end)


def test_front_end_restart_from_populations_file(lbmc, tmp_path):
    path, arrays = channel(tmp_path, lx=32, ly=24, extra="MaxT 300\nFileOut 300\nSteadyCheck 0\n")
    with engine(lbmc, 32, 24, arrays) as eng:
        eng.iterate(201, lbmc.SYNC)
        f_mid = eng.f()
        eng.iterate(300, lbmc.STORE_MACROS | lbmc.SYNC)
        u_end = eng.u()
    np.save(tmp_path / "dom" / "Populations.npy", f_mid)
    text = open(path).read() + "Init 2\n"
    open(path, "w").write(text)
    st, res = lbmc.run(path, storage="f32")
    assert st == lbmc.OK and res.steps == 300
    np.testing.assert_array_equal(load_solution(tmp_path / "out", 300)["VelocityX"], u_end[0])
