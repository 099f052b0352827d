"""Pins the engine's input-file reader (lbmc_read_input) to the reference's
own InfileReader (LBM-C/infile_reader.cu:45-226), host-compiled from the
reference sources by oracle/build_ref.sh into oracle/_ref/libref_reader_*.so.

Both readers parse the same files; every field the file sets must come out
equal (bit for bit for numbers: this is parsing).  The reference fixes the
lattice at compile time (macros.cu:11-12), so 2-D files go to the D2Q9
build and 3-D files to the D3Q15 build; the engine picks the lattice from
Lz.  Fields a file does not set are not compared: the reference leaves them
uninitialised, the engine keeps lbmc_config_default's values.
CPU only."""
import ctypes
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


class RefInput(ctypes.Structure):
    """struct ref_input of oracle/ref_reader_shim.cpp (STR_LENGTH = 64)."""
    _fields_ = [("tau", ctypes.c_double), ("tau_mrt", ctypes.c_double * 15),
                ("c_smag", ctypes.c_double), ("tolerance", ctypes.c_double),
                ("length", ctypes.c_int * 3), ("h", ctypes.c_int), ("dt", ctypes.c_int),
                ("forcing", ctypes.c_int), ("macro_bc", ctypes.c_int), ("micro_bc", ctypes.c_int),
                ("collision_type", ctypes.c_int), ("init_type", ctypes.c_int),
                ("max_t", ctypes.c_int), ("plot", ctypes.c_int), ("screen", ctypes.c_int),
                ("steady_check", ctypes.c_int), ("out_u", ctypes.c_int * 3),
                ("out_rho", ctypes.c_int), ("out_pressure", ctypes.c_int),
                ("interactive", ctypes.c_int), ("screen_node", ctypes.c_int * 3),
                ("name", ctypes.c_char * 64), ("domain_fname", ctypes.c_char * 64),
                ("output_fname", ctypes.c_char * 64)]


def ref_reader(lattice):
    path = os.path.join(REF_DIR, f"libref_reader_{lattice}.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref reader not built (needs the reference sources)")
    lib = ctypes.CDLL(path)
    lib.ref_read_input.argtypes = [ctypes.c_char_p, ctypes.POINTER(RefInput), ctypes.c_char_p,
                                   ctypes.c_size_t]
    assert lib.ref_reader_str_length() == 64
    return lib


def read_both(lbmc, path, lattice):
    lib = ref_reader(lattice)
    ref = RefInput()
    report = ctypes.create_string_buffer(1 << 16)
    dim = lib.ref_read_input(os.fsencode(path), ctypes.byref(ref), report, len(report))
    assert dim == (2 if lattice == "d2q9" else 3)
    rc, echo = lbmc.read_input(path)
    return ref, rc, report.value.decode(), echo


# key -> (reference field(s), engine getter)
def fields(ref, rc, dim, q):
    c = rc.cfg
    return {
        "ProjName": (ref.name, rc.project_name),
        "DomainFile": (ref.domain_fname, rc.domain_file),
        "OutputFile": (ref.output_fname, rc.output_file),
        "TauMRT": (list(ref.tau_mrt)[:q], list(c.tau_mrt)[:q]),
        "Tau": (ref.tau, c.tau),
        "Lx": (ref.length[0], c.length[0]),
        "Ly": (ref.length[1], c.length[1]),
        "Lz": (ref.length[2], c.length[2]) if dim == 3 else (None, None),
        "DeltaX": (ref.h, c.h),
        "DeltaT": (ref.dt, c.dt),
        "C_smag": (ref.c_smag, c.c_smag),
        "ColType": (ref.collision_type, c.collision_type),
        "Force": (ref.forcing, c.forcing),
        "MicroBC": (ref.micro_bc, c.micro_bc),
        "MacroBC": (ref.macro_bc, c.macro_bc),
        "Tolerance": (ref.tolerance, c.tolerance),
        "Init": (ref.init_type, c.init_type),
        "MaxT": (ref.max_t, rc.max_t),
        "FileOut": (ref.plot, rc.file_out),
        "ScreenMes": (ref.screen, rc.screen_mes),
        "SteadyCheck": (ref.steady_check, rc.steady_check),
        "OutputVars": ([*list(ref.out_u)[:dim], ref.out_rho, ref.out_pressure],
                       [*list(rc.output_u)[:dim], rc.output_rho, rc.output_pressure]),
        "ScreenNode": (list(ref.screen_node)[:dim], list(rc.screen_node)[:dim]),
        "Interactive": (ref.interactive, rc.interactive),
    }


def assert_same(ref, rc, keys, dim, q):
    f = fields(ref, rc, dim, q)
    for k in keys:
        a, b = f[k]
        if isinstance(a, float):
            assert np.float64(a).tobytes() == np.float64(b).tobytes(), (k, a, b)
        else:
            assert a == b, (k, a, b)


FULL = """\
# the reference's example layout
ProjName      {name}   # trailing comment
DomainFile    dom_{name}
OutputFile    out_{name}
Tau           0.8
TauMRT        {mrt}
Lx            128
Ly            64
Lz            {lz}
DeltaX        1
DeltaT        1
C_smag        0.13
ColType       {col}
Force         1
MicroBC       1
MacroBC       0
Tolerance     1e-9
Init          0
MaxT          2000
FileOut       500
ScreenMes     100
SteadyCheck   50
OutputVars    1 0 1 1 0
ScreenNode    64 32 {nz}
Interactive   0
this line is echoed
"""

ALL_KEYS = ["ProjName", "DomainFile", "OutputFile", "TauMRT", "Tau", "Lx", "Ly", "Lz", "DeltaX",
            "DeltaT", "C_smag", "ColType", "Force", "MicroBC", "MacroBC", "Tolerance", "Init",
            "MaxT", "FileOut", "ScreenMes", "SteadyCheck", "OutputVars", "ScreenNode",
            "Interactive"]


@pytest.mark.parametrize("lattice", ["d2q9", "d3q15"])
@pytest.mark.parametrize("col", ["BGK", "NTPOR", "MRT", "MRTPOR", "NTPOR MRT", "MRT BGK"])
def test_full_files_parse_alike(lbmc, tmp_path, lattice, col):
    dim, q = (2, 9) if lattice == "d2q9" else (3, 15)
    mrt = " ".join(f"{1 + 0.013 * i:.3f}" for i in range(q))
    text = FULL.format(name="run_" + lattice, mrt=mrt, lz=1 if dim == 2 else 48, col=col,
                       nz=0 if dim == 2 else 7)
    path = tmp_path / "in.txt"
    path.write_text(text)
    ref, rc, report, echo = read_both(lbmc, str(path), lattice)
    assert rc.cfg.lattice == (lbmc.D2Q9 if dim == 2 else lbmc.D3Q15)
    assert_same(ref, rc, ALL_KEYS, dim, q)
    # the unknown line is echoed by both
    assert "this line is echoed" in report and "this line is echoed" in echo


EDGE = [
    # (name, lattice, text, keys compared)
    ("duplicate keys: the last wins", "d2q9", "Lx 10\nLy 12\nTau 0.6\nTau 0.75\nLx 14\n",
     ["Lx", "Ly", "Tau"]),
    ("key inside a longer word", "d2q9", "Taux 0.55\nLxx 9\nLy 3\n", ["Tau", "Lx", "Ly"]),
    ("leading blanks and tabs", "d3q15", "   Tau\t0.71\n\tLx 5\n  Ly 6\nLz 7\n",
     ["Tau", "Lx", "Ly", "Lz"]),
    ("a key in a comment only", "d2q9", "Lx 4 # Tau 0.9\nLy 4\n# Tau 0.6\nTau 0.8\n",
     ["Lx", "Ly", "Tau"]),
    ("extra tokens after the value", "d3q15", "Tau 0.7 0.9 junk\nLx 8 9\nLy 4\nLz 2\nMaxT 100 200\n",
     ["Tau", "Lx", "Ly", "Lz", "MaxT"]),
    ("scientific and signed numbers", "d2q9", "Tolerance 2.5E-7\nC_smag +0.1\nTau 8e-1\nLx 4\nLy 4\n",
     ["Tolerance", "C_smag", "Tau", "Lx", "Ly"]),
    ("ProjName before Tau, OutputFile before Force", "d2q9",
     "ProjName TauCase\nOutputFile Force_run\nLx 4\nLy 4\n", ["ProjName", "OutputFile", "Lx", "Ly"]),
    ("2-D build ignores Lz and the third OutputVars and ScreenNode values", "d2q9",
     "Lx 6\nLy 5\nLz 1\nOutputVars 1 1 1 0 1\nScreenNode 3 2 1\n",
     ["Lx", "Ly", "OutputVars", "ScreenNode"]),
    ("3-D OutputVars and ScreenNode take z", "d3q15",
     "Lx 6\nLy 5\nLz 4\nOutputVars 0 1 1 1 1\nScreenNode 3 2 1\n",
     ["Lx", "Ly", "Lz", "OutputVars", "ScreenNode"]),
    ("Interactive and Init", "d3q15", "Lx 2\nLy 2\nLz 2\nInteractive 1\nInit 1\n",
     ["Interactive", "Init"]),
    ("ColType without a known name keeps the default", "d2q9", "Lx 2\nLy 2\nColType 0\n", []),
    # stream-extraction semantics of the reference's `stringstream >> field`
    ("bool fields from integers other than 0/1", "d2q9",
     "Lx 4\nLy 4\nForce 2\nMacroBC -1\nInteractive 2\n", ["Force", "MacroBC", "Interactive"]),
    ("bool field from a word", "d2q9", "Lx 4\nLy 4\nForce true\n", ["Force"]),
    ("a non-numeric value", "d2q9", "Lx 4\nLy 4\nMaxT abc\n", ["MaxT"]),
    ("a number followed by letters", "d2q9", "Lx 4\nLy 4\nTau 0.8abc\n", ["Tau"]),
    ("a fractional integer field", "d2q9", "Lx 4.7\nLy 4\n", ["Lx", "Ly"]),
    ("fewer TauMRT values than Q", "d2q9", "Lx 4\nLy 4\nTauMRT 1 2 3\n", ["TauMRT"]),
    ("fewer OutputVars values than five", "d2q9", "Lx 4\nLy 4\nOutputVars 1 1\n", ["OutputVars"]),
]


@pytest.mark.parametrize("name,lattice,text,keys", EDGE, ids=[e[0] for e in EDGE])
def test_edge_cases_parse_alike(lbmc, tmp_path, name, lattice, text, keys):
    dim, q = (2, 9) if lattice == "d2q9" else (3, 15)
    path = tmp_path / "in.txt"
    path.write_text(text)
    ref, rc, _, _ = read_both(lbmc, str(path), lattice)
    assert_same(ref, rc, keys, dim, q)


@pytest.mark.parametrize("lattice", ["d2q9", "d3q15"])
def test_tau_mrt_reads_q_values(lbmc, tmp_path, lattice):
    """TauMRT takes the lattice's Q values; a line with more keeps the first Q."""
    dim, q = (2, 9) if lattice == "d2q9" else (3, 15)
    vals = " ".join(f"{0.5 + 0.1 * i:g}" for i in range(15))
    lz = "Lz 3\n" if dim == 3 else ""
    path = tmp_path / "in.txt"
    path.write_text(f"Lx 3\nLy 3\n{lz}TauMRT {vals}\n")
    ref, rc, _, _ = read_both(lbmc, str(path), lattice)
    assert_same(ref, rc, ["TauMRT"], dim, q)
