"""Run-control front end on the CPU: the input-file reader against the
reference's key semantics (LBM-C/infile_reader.cu:45-226), the domain
loader (LBM-C/model_builder.cu:173-231 field names) and the
CGNS-structured output writer.  No GPU is touched."""
import ctypes
import json
import os

import numpy as np
import pytest

FULL_2D = """\
# channel flow, the reference's example layout
ProjName      channel   # trailing comment
DomainFile    {dom}
OutputFile    {out}
Tau           0.8
TauMRT        1.0 1.19 1.19 1.0 1.2 1.0 1.2 1.25 1.25
Lx            128
Ly            64
Lz            1
DeltaX        1
DeltaT        1
C_smag        0.0
ColType       BGK
Force         1
MicroBC       0
MacroBC       0
Tolerance     1e-9
Init          0
MaxT          2000
FileOut       500
ScreenMes     100
SteadyCheck   50
OutputVars    1 1 1 1 0
ScreenNode    64 32 0
Interactive   0
this line is echoed
"""


def write(tmp_path, text, name="input.txt"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_reader_full_2d(lbmc, tmp_path):
    path = write(tmp_path, FULL_2D.format(dom=tmp_path / "dom", out=tmp_path / "out"))
    rc, echo = lbmc.read_input(path)
    c = rc.cfg
    assert rc.project_name == b"channel"
    assert rc.domain_file == str(tmp_path / "dom").encode()
    assert c.lattice == lbmc.D2Q9 and tuple(c.length) == (128, 64, 1)
    assert c.tau == 0.8 and rc.tau_mrt_count == 9
    assert list(c.tau_mrt)[:9] == [1.0, 1.19, 1.19, 1.0, 1.2, 1.0, 1.2, 1.25, 1.25]
    assert c.collision_type == lbmc.BGK and c.forcing == 1 and c.micro_bc == 0 and c.macro_bc == 0
    assert c.tolerance == 1e-9 and c.init_type == 0 and c.h == 1 and c.dt == 1
    assert (rc.max_t, rc.file_out, rc.screen_mes, rc.steady_check) == (2000, 500, 100, 50)
    assert list(rc.output_u) == [1, 1, 0] and rc.output_rho == 1 and rc.output_pressure == 0
    assert list(rc.screen_node)[:2] == [64, 32] and rc.interactive == 0
    assert "Tau = 0.8" in echo and "S_8 = 1.25" in echo and "ColType = BGK" in echo
    assert "this line is echoed" in echo


def test_reader_3d_and_lattice_choice(lbmc, tmp_path):
    text = ("Lx 24\nLy 16\nLz 12\nTau 0.7\nColType MRTPOR\nOutputVars 1 1 1 1 0\n"
            "ScreenNode 1 2 3\nTauMRT " + " ".join(["1.1"] * 15) + "\n")
    rc, _ = lbmc.read_input(write(tmp_path, text))
    assert rc.cfg.lattice == lbmc.D3Q15 and tuple(rc.cfg.length) == (24, 16, 12)
    assert rc.cfg.collision_type == lbmc.MRTPOR  # "MRTPOR" contains "MRT": last match wins
    assert list(rc.output_u) == [1, 1, 1] and list(rc.screen_node) == [1, 2, 3]
    assert rc.tau_mrt_count == 15
    # Lz 1 (or none): D2Q9, z ignored as in a 2-D build of the reference.
    rc, _ = lbmc.read_input(write(tmp_path, "Lx 8\nLy 8\nLz 1\nOutputVars 1 1 1 1 0\n", "b.txt"))
    assert rc.cfg.lattice == lbmc.D2Q9 and rc.cfg.length[2] == 1 and rc.output_u[2] == 0
    # The extension key overrides.
    rc, _ = lbmc.read_input(write(tmp_path, "Lattice D3Q15\nLx 8\nLy 8\nLz 1\n", "c.txt"))
    assert rc.cfg.lattice == lbmc.D3Q15


@pytest.mark.parametrize("line,field,value", [
    ("ColType NTPOR", "collision_type", 1), ("ColType MRT", "collision_type", 2),
    ("ColType BGK", "collision_type", 0),
    ("Tau 0.6 # TauMRT is ignored in a comment", "tau", 0.6),
    ("C_smag 0.17", "c_smag", 0.17), ("Init 1", "init_type", 1),
    ("MacroBC 1", "macro_bc", 1), ("MicroBC 1", "micro_bc", 1),
])
def test_reader_single_keys(lbmc, tmp_path, line, field, value):
    rc, _ = lbmc.read_input(write(tmp_path, "Lx 4\nLy 4\n" + line + "\n"))
    assert getattr(rc.cfg, field) == pytest.approx(value)


def test_reader_key_order_is_the_references(lbmc, tmp_path):
    # Keys are matched by substring in the reference's order, values
    # included: "ProjName" is tried before "Tau", so a project named TauCase
    # is a project name; "OutputFile" before "Force".
    rc, _ = lbmc.read_input(write(tmp_path, "ProjName TauCase\nOutputFile Force_run\nLx 4\nLy 4\n"))
    assert rc.project_name == b"TauCase" and rc.output_file == b"Force_run"
    assert rc.cfg.tau == 1.0 and rc.cfg.forcing == 0


def test_reader_missing_file(lbmc, tmp_path):
    with pytest.raises(lbmc.LbmcError) as e:
        lbmc.read_input(str(tmp_path / "nope.txt"))
    assert e.value.status == lbmc.ERR_IO


def model_arrays(lbmc, rc):
    lib = lbmc.library()
    h = ctypes.c_void_p()
    lbmc.check(lib.lbmc_model_build(ctypes.byref(rc), ctypes.byref(h)))
    dom = lbmc.Domain()
    lbmc.check(lib.lbmc_model_domain(h, ctypes.byref(dom)))
    n = rc.cfg.length[0] * rc.cfg.length[1] * rc.cfg.length[2]

    def arr(p, ct, count=n):
        return None if not p else np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ct)), (count,)).copy()
    out = dict(geometry=arr(dom.geometry, ctypes.c_double),
               force=[arr(dom.force[d], ctypes.c_double) for d in range(3)],
               u=[arr(dom.u[d], ctypes.c_double) for d in range(3)], rho=arr(dom.rho, ctypes.c_double),
               macro=arr(dom.macro_bc, ctypes.c_int), micro=arr(dom.micro_bc, ctypes.c_int))
    lib.lbmc_model_free(h)
    return out


def test_model_builder_reads_fields(lbmc, tmp_path):
    dom = tmp_path / "dom"
    dom.mkdir()
    lx, ly = 6, 5
    n = lx * ly
    rng = np.random.default_rng(0)
    por = (rng.random((ly, lx)) < 0.2).astype(np.float32)       # float32 on disk
    fx, fy = rng.random(n), rng.random(n)
    macro = rng.integers(0, 3, n).astype(np.int64)              # int64 on disk
    micro = rng.integers(0, 2, n).astype(np.int32)
    ux, uy, rho = rng.random(n), rng.random(n), 1 + rng.random(n)
    for name, a in dict(Porosity=por, ForceX=fx, ForceY=fy, MacroBC=macro, MicroBC=micro,
                        VelocityX=ux, VelocityY=uy, Rho=rho).items():
        np.save(dom / f"{name}.npy", a)
    path = write(tmp_path, f"DomainFile {dom}\nLx {lx}\nLy {ly}\nForce 1\nMacroBC 1\nMicroBC 1\n")
    rc, _ = lbmc.read_input(path)
    m = model_arrays(lbmc, rc)
    np.testing.assert_array_equal(m["geometry"], por.reshape(-1))
    np.testing.assert_array_equal(m["force"][0], fx)
    np.testing.assert_array_equal(m["force"][1], fy)
    np.testing.assert_array_equal(m["macro"], macro)
    np.testing.assert_array_equal(m["micro"], micro)
    np.testing.assert_array_equal(m["u"][0], ux)
    np.testing.assert_array_equal(m["rho"], rho)
    assert m["u"][2] is None and m["force"][2] is None


def test_model_builder_errors(lbmc, tmp_path):
    dom = tmp_path / "dom"
    dom.mkdir()
    path = write(tmp_path, f"DomainFile {dom}\nLx 4\nLy 4\nForce 1\n")
    rc, _ = lbmc.read_input(path)
    h = ctypes.c_void_p()
    st = lbmc.library().lbmc_model_build(ctypes.byref(rc), ctypes.byref(h))
    assert st == lbmc.ERR_IO and b"ForceX" in lbmc.library().lbmc_last_error()
    np.save(dom / "ForceX.npy", np.zeros(15))  # wrong size
    np.save(dom / "ForceY.npy", np.zeros(16))
    st = lbmc.library().lbmc_model_build(ctypes.byref(rc), ctypes.byref(h))
    assert st == lbmc.ERR_IO and b"expected 16" in lbmc.library().lbmc_last_error()
    # No Porosity file: all fluid (geometry NULL).
    np.save(dom / "ForceX.npy", np.zeros(16))
    m = model_arrays(lbmc, rc)
    assert m["geometry"] is None


@pytest.mark.parametrize("dim,length", [(2, (5, 3)), (3, (4, 3, 2))])
def test_output_tree(lbmc, tmp_path, dim, length):
    out = tmp_path / "out"
    n = int(np.prod(length))
    o = lbmc.Output(str(out), dim, length)
    a, b = np.arange(n, dtype=float), -np.arange(n, dtype=float)
    o.append(100, {"VelocityX": a, "Density": b})
    o.append(200, {"VelocityX": b})
    o.close()
    idx = json.loads((out / "index.json").read_text())
    base = idx["Base"]
    zone = base["Zone"]
    assert base["name"] == "Base" and zone["name"] == "LBM-C Output Data"
    assert zone["vertex_size"] == [x + 1 for x in length] and zone["cell_size"] == list(length)
    assert base["BaseIterativeData"]["IterationValues"] == [100, 200]
    assert zone["ZoneIterativeData"]["FlowSolutionPointers"] == ["Solution @ Time = 100",
                                                                  "Solution @ Time = 200"]
    assert idx["complete"] is True
    sol = zone["FlowSolutions"][0]
    assert sol["GridLocation"] == "CellCenter" and set(sol["fields"]) == {"VelocityX", "Density"}
    vx = np.load(out / sol["fields"]["VelocityX"])
    assert vx.shape == tuple(reversed(length)) and vx.dtype == np.float64
    np.testing.assert_array_equal(vx.reshape(-1), a)
    cx = np.load(out / "GridCoordinates" / "CoordinateX.npy")
    assert cx.dtype == np.float32 and cx.shape == tuple(x + 1 for x in reversed(length))
    assert cx.reshape(-1)[:length[0] + 1].tolist() == list(range(length[0] + 1))
