"""The infraga-accel-* front ends: the reference's MPI build names
(src/main.infraga.*.mpi.cpp), as run_infraga.py launches them with
`mpirun -np N` for --cpu-cnt N >= 2.  The first process traces the whole job on
the GPU and writes the serial binaries' files under the accel header (the
`threads` line of the MPI summaries); later ranks of the launch exit at once;
source and receiver lists (srcs_list= / rcvrs_list=) give one arrivals file per
pair, named as the MPI build names them, each with the rows of the serial
search for that pair."""
import os
import subprocess
import tempfile

import pytest

from tests._cases import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "bin")


@pytest.fixture(scope="module")
def built():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    for b in ("infraga-3d", "infraga-accel-3d", "infraga-accel-sph", "infraga-accel-3d-rngdep",
              "infraga-accel-sph-rngdep"):
        assert os.path.exists(os.path.join(BIN, b)), f"bin/{b} missing: run __graft_entry__.build()"
    return True


def _run(work, binary, argv, env=None):
    e = dict(os.environ)
    e.update(env or {})
    subprocess.run([os.path.join(BIN, binary), *argv], cwd=work, stdin=subprocess.DEVNULL, stdout=subprocess.DEVNULL,
                   check=True, timeout=600, env=e)


def _stage(work):
    import shutil
    shutil.copy(os.path.join(GOLDEN, "profiles", "gen0.met"), os.path.join(work, "atmo.met"))


def _body(text):
    return [ln for ln in text.splitlines() if ln.strip() and not ln.startswith("#")]


def test_accel_prop_equals_serial(built):
    argv = ["-prop", "atmo.met", "incl_min=5", "incl_max=25", "incl_step=5", "az_min=0", "az_max=90", "az_step=90",
            "bounces=2", "max_rng=600", "write_rays=false"]
    with tempfile.TemporaryDirectory() as w1, tempfile.TemporaryDirectory() as w2:
        _stage(w1); _stage(w2)
        _run(w1, "infraga-3d", argv)
        _run(w2, "infraga-accel-3d", argv, env={"OMPI_COMM_WORLD_RANK": "0", "OMPI_COMM_WORLD_SIZE": "4"})
        a = open(os.path.join(w1, "atmo.arrivals.dat")).read()
        b = open(os.path.join(w2, "atmo.arrivals.dat")).read()
    assert "# infraga-accel-3d -prop summary:" in b and "#\tthreads: 4" in b
    assert _body(a) == _body(b) and len(_body(a)) > 2


def test_accel_later_ranks_exit(built):
    with tempfile.TemporaryDirectory() as w:
        _stage(w)
        _run(w, "infraga-accel-3d", ["-prop", "atmo.met", "inclination=10", "azimuth=90"],
             env={"OMPI_COMM_WORLD_RANK": "2", "OMPI_COMM_WORLD_SIZE": "4"})
        assert sorted(os.listdir(w)) == ["atmo.met"]


def test_accel_receiver_list_matches_single_searches(built):
    rcvrs = [(250.0, 40.0), (-180.0, 120.0)]
    common = ["bnc_min=0", "bnc_max=1", "incl_min=5", "incl_max=30"]
    with tempfile.TemporaryDirectory() as w:
        _stage(w)
        with open(os.path.join(w, "rcvrs.dat"), "w") as f:
            for x, y in rcvrs:
                f.write(f"{x} {y}\n")
        _run(w, "infraga-accel-3d", ["-eig_search", "atmo.met", "rcvrs_list=rcvrs.dat", *common])
        listed = [open(os.path.join(w, f"atmo.rcvr-{i}.arrivals.dat")).read() for i in range(len(rcvrs))]
        singles = []
        for i, (x, y) in enumerate(rcvrs):
            _run(w, "infraga-3d", ["-eig_search", "atmo.met", f"rcvr_x={x}", f"rcvr_y={y}", *common,
                                   f"output_id=single{i}"])
            singles.append(open(os.path.join(w, f"single{i}.arrivals.dat")).read())
        n_paths = [len([f for f in os.listdir(w) if f.startswith(f"atmo.rcvr-{i}.eigenray-")]) for i in range(2)]
    for i in range(len(rcvrs)):
        assert "# infraga-accel-3d -eig_search summary:" in listed[i]
        assert _body(listed[i]) == _body(singles[i])
        assert n_paths[i] == len(_body(singles[i]))
    assert sum(n_paths) > 0
