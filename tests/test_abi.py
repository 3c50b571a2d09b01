"""The C ABI: the library loads and exports every entry point include/mdb.h
declares, and the ctypes mirror matches the header.  No compute calls: these
run without a GPU."""

from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def header_functions() -> list[str]:
    text = (ROOT / "include" / "mdb.h").read_text()
    return sorted(set(re.findall(r"^(?:int|const char\*|void)\s+(mdb_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    import importlib.util
    import sys

    spec = importlib.util.spec_from_file_location("mdb_build", ROOT / "making-it-rain-webgpu_b200" / "build.py")
    build = importlib.util.module_from_spec(spec)
    sys.modules["mdb_build"] = build
    spec.loader.exec_module(build)
    build.build()
    from mdb200 import abi

    return abi.load()


def test_header_declares_the_boundary():
    names = header_functions()
    for want in ("mdb_create", "mdb_batch_create", "mdb_run", "mdb_evaluate", "mdb_potential",
                 "mdb_get_positions", "mdb_set_box", "mdb_destroy", "mdb_last_error"):
        assert want in names


def test_library_exports_every_declared_symbol(lib):
    for name in header_functions():
        assert hasattr(lib, name), name


def test_ctypes_mirror_covers_the_header():
    from mdb200 import abi

    assert set(abi.EXPORTS) == set(header_functions())


def test_abi_version_and_status_strings(lib):
    from mdb200 import abi

    assert lib.mdb_abi_version() == abi.ABI_VERSION
    assert lib.mdb_status_string(abi.ERR_CUTOFF_TOO_LARGE_FOR_BOX) == b"cutoff too large for box"
    assert lib.mdb_status_string(12345) == b"unknown status"


def test_struct_layouts_match_the_header():
    """Field offsets the C compiler would give, checked by ctypes arithmetic."""
    from mdb200 import abi

    assert C.sizeof(abi.Energies) == 8 * (18 + 9 + 1 + 9)
    assert abi.SystemDesc.box.offset == 16
    assert abi.StateDesc.box.offset == 16
    assert abi.RunOptions.seed.offset == 32


def test_null_arguments_are_refused_without_a_device(lib):
    from mdb200 import abi

    assert lib.mdb_create(None, None, None, None) == abi.ERR_INVALID_ARGUMENT
    assert lib.mdb_run(None, 1) == abi.ERR_INVALID_ARGUMENT
    assert lib.mdb_destroy(None, None) == abi.ERR_INVALID_ARGUMENT
    assert lib.mdb_last_error(None) == b"no engine"


def test_every_struct_mirror_matches_the_c_compiler(tmp_path):
    """sizeof and every field offset of the header's structs, from gcc, against
    the ctypes mirrors the Python host side passes to the library."""
    import shutil
    import subprocess

    from mdb200 import abi

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    mirrors = {"mdb_tuning": abi.Tuning, "mdb_run_options": abi.RunOptions, "mdb_energies": abi.Energies,
               "mdb_barostat_stats": abi.BarostatStats, "mdb_profile": abi.Profile,
               "mdb_neighbour_stats": abi.NeighbourStats, "mdb_system_desc": abi.SystemDesc,
               "mdb_state_desc": abi.StateDesc}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "mdb.h"', "int main(void) {"]
    for cname, mirror in mirrors.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for field, _ in mirror._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("  return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    include = ROOT / "include"
    subprocess.run(["gcc", "-std=c11", "-I", str(include), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            cname, field, value = line.split()
            got[(cname, field)] = int(value)
    for cname, mirror in mirrors.items():
        assert got[(cname, "sizeof")] == C.sizeof(mirror), cname
        for field, _ in mirror._fields_:
            assert got[(cname, field)] == getattr(mirror, field).offset, (cname, field)


def test_node_addon_exports_what_the_typescript_shim_calls():
    """The TypeScript StepLoop's addon interface and the Node-API addon's
    export table name the same methods, and the addon calls only entry points
    the header declares (neither can be built here: no Node)."""
    ts = (ROOT / "making-it-rain-webgpu_b200" / "ts" / "step-loop.ts").read_text()
    cc = (ROOT / "making-it-rain-webgpu_b200" / "napi" / "addon.cc").read_text()
    header = (ROOT / "include" / "mdb.h").read_text()
    block = ts[ts.index("interface MdbAddon {"):]
    block = block[:block.index("\n}")]
    wanted = set(re.findall(r"^\s+(\w+)\(", block, re.M))
    exported = set(re.findall(r'\{"(\w+)", nullptr, \w+,', cc))
    assert wanted == exported, (wanted ^ exported)
    called = set(re.findall(r"\b(mdb_[a-z_]+)\(", cc))
    declared = set(re.findall(r"\b(mdb_[a-z_]+)\(", header))
    assert called <= declared, called - declared


C_CLIENT = r"""
#include <stdio.h>
#include <string.h>
#include "mdb.h"

/* A C caller of the library: version, argument checks, the reference's named
   errors (found on the host, before any device work), and one engine whose
   creation must stop at the device check on a machine without a GPU. */
int main(void) {
  if (mdb_abi_version() != MDB_ABI_VERSION) return 1;
  mdb_engine* e = NULL;
  if (mdb_create(NULL, NULL, NULL, &e) != MDB_ERR_INVALID_ARGUMENT) return 2;
  static const double masses[3] = {15.99943, 1.007947, 1.007947};
  static const double pos[9] = {1.0, 1.0, 1.0, 1.09572, 1.0, 1.0, 0.97600, 1.09267, 1.0};
  static const double charge[3] = {-0.834, 0.417, 0.417}, sigma[3] = {0.315, 1.0, 1.0},
                      epsilon[3] = {0.636, 0.0, 0.0};
  static const int32_t ex1[3] = {0, 0, 1}, ex2[3] = {1, 2, 2};
  static const double exq[3] = {0.0, 0.0, 0.0}, exs[3] = {1.0, 1.0, 1.0}, exe[3] = {0.0, 0.0, 0.0};
  mdb_system_desc sys;
  memset(&sys, 0, sizeof sys);
  sys.n_particles = 3;
  sys.masses = masses;
  sys.box[0] = sys.box[4] = sys.box[8] = 3.0;
  mdb_state_desc st;
  memset(&st, 0, sizeof st);
  st.positions = pos;
  st.box[0] = st.box[4] = st.box[8] = 3.0;
  mdb_run_options opt;
  memset(&opt, 0, sizeof opt);
  int rc = mdb_create(&sys, &st, &opt, &e); /* time step 0 */
  printf("%d %s\n", rc, mdb_last_error(e));
  if (rc != MDB_ERR_INVALID_ARGUMENT) return 3;
  mdb_destroy(e, NULL);
  opt.time_step = 0.002;
  opt.temperature = 300.0;
  opt.friction = 1.0;
  rc = mdb_create(&sys, &st, &opt, &e); /* no NonbondedForce */
  printf("%d %s\n", rc, mdb_last_error(e));
  if (rc != MDB_ERR_UNSUPPORTED_FORCE) return 8;
  mdb_destroy(e, NULL);
  sys.has_nonbonded = 1;
  sys.cutoff = 1.6; /* more than half the 3 nm box */
  sys.ewald_tolerance = 5e-4;
  sys.use_dispersion_correction = 1;
  sys.charge = charge;
  sys.sigma = sigma;
  sys.epsilon = epsilon;
  sys.n_exceptions = 3;
  sys.exception_p1 = ex1;
  sys.exception_p2 = ex2;
  sys.exception_charge_prod = exq;
  sys.exception_sigma = exs;
  sys.exception_epsilon = exe;
  rc = mdb_create(&sys, &st, &opt, &e);
  printf("%d %s\n", rc, mdb_last_error(e));
  if (rc != MDB_ERR_CUTOFF_TOO_LARGE_FOR_BOX) return 9;
  mdb_destroy(e, NULL);
  sys.cutoff = 1.0;
  opt.mesh[0] = opt.mesh[1] = opt.mesh[2] = 22; /* 2 x 11: not 2/3/5/7-smooth */
  rc = mdb_create(&sys, &st, &opt, &e);
  printf("%d %s\n", rc, mdb_last_error(e));
  if (rc != MDB_ERR_NOT_SMOOTH) return 10;
  mdb_destroy(e, NULL);
  opt.mesh[0] = opt.mesh[1] = opt.mesh[2] = 0;
  e = NULL;
  rc = mdb_create(&sys, &st, &opt, &e);
  printf("%d %s\n", rc, mdb_last_error(e));
  int64_t leaked = -1;
  if (e && mdb_destroy(e, &leaked) != MDB_OK) return 4;
  if (leaked != 0) return 5;
  return rc == MDB_ERR_NO_DEVICE ? 0 : rc == MDB_OK ? 7 : 6;
}
"""


def test_a_c_program_links_the_library(tmp_path):
    """The header is plain C11 (warnings are errors) and a C program links
    libmdb200.so and gets the documented status codes: the reference's named
    errors for a System without a NonbondedForce, a cutoff past half the box
    and a mesh that is not 2/3/5/7-smooth come from the host checks, before
    any device work.  Without a GPU the valid engine stops at the device
    check; with one it is created and destroyed."""
    import shutil
    import subprocess

    from mdb200 import abi

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    lib_path = abi.LIBRARY_PATH
    if not lib_path.exists():
        pytest.skip("library not built")
    src = tmp_path / "client.c"
    src.write_text(C_CLIENT)
    exe = tmp_path / "client"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"), str(src),
                    "-L", str(lib_path.parent), "-lmdb200", f"-Wl,-rpath,{lib_path.parent}", "-o", str(exe)],
                   check=True)
    run = subprocess.run([str(exe)], capture_output=True, text=True)
    if run.returncode == 7:
        pytest.skip("a device is visible: the engine was created")
    assert run.returncode == 0, (run.returncode, run.stdout)
    assert "time_step must be positive" in run.stdout
    assert "NonbondedForce" in run.stdout
    assert "cutoff does not fit this box" in run.stdout
    assert "not 2/3/5/7-smooth" in run.stdout
    assert "no CUDA device is visible" in run.stdout


def test_named_errors_reach_python_before_any_device_work():
    """The reference's named errors (system.ts:178, triclinic.ts:179,
    constraint-clusters.ts:71, fft.ts:24) come from the engine's host checks,
    so the Python mirror raises them on any machine."""
    import dataclasses

    import numpy as np

    from mdb200 import steploop, synth

    system, state = synth.water_box(n_waters=100, width=1.5, seed=1, grid=(16, 16, 16))
    with pytest.raises(steploop.CutoffTooLargeForBox, match="cutoff does not fit this box"):
        steploop.StepLoop.from_parsed(system, state, steploop.RunOptions())

    system, state = synth.water_box(n_waters=300, width=2.1, seed=5)
    with pytest.raises(steploop.NotSmooth, match="not 2/3/5/7-smooth"):
        steploop.StepLoop.from_parsed(system, state, steploop.RunOptions(mesh=(22, 22, 22)))

    # chain the first five waters' oxygens: one constraint cluster of 15 atoms
    oxygens = np.arange(0, 15, 3, dtype=np.int32)
    chained = dataclasses.replace(
        system,
        constraint_p1=np.concatenate([system.constraint_p1, oxygens[:-1]]).astype(np.int32),
        constraint_p2=np.concatenate([system.constraint_p2, oxygens[1:]]).astype(np.int32),
        constraint_distance=np.concatenate([system.constraint_distance,
                                            np.linalg.norm(state.positions[oxygens[1:]]
                                                           - state.positions[oxygens[:-1]], axis=1)]))
    with pytest.raises(steploop.ClusterTooLarge):
        steploop.StepLoop.from_parsed(chained, state, steploop.RunOptions())


def test_mesh_axes_shorter_than_the_spline_are_refused_before_device_work(lib):
    """An order-5 B-spline spans five mesh points, wrapped once into the mesh,
    so an axis of fewer than five points is refused on the host: by the engine
    (as an invalid argument) and by the allocation-free reciprocal-space entry
    point, before either touches a device."""
    import numpy as np

    from mdb200 import abi, steploop, synth

    system, state = synth.water_box(n_waters=300, width=2.1, seed=5)
    with pytest.raises(steploop.EngineError, match="below the 5 points"):
        steploop.StepLoop.from_parsed(system, state, steploop.RunOptions(mesh=(24, 3, 24)))

    box = np.ascontiguousarray((np.eye(3) * 3.0).reshape(9))
    dummy = C.c_void_p(1)  # never dereferenced: the size check comes first
    for axes in ((3, 16, 16), (16, 4, 16), (16, 16, 2)):
        mesh = (C.c_int32 * 3)(*axes)
        status = lib.mdb_reciprocal_noalloc(1, dummy, dummy, box.ctypes.data_as(C.POINTER(C.c_double)), 3.0, mesh,
                                            dummy, dummy, None)
        assert status == abi.ERR_INVALID_ARGUMENT, (axes, status)
