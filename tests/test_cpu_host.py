"""CPU-side checks of the product: the C ABI library loads and exports every
entry point declared in include/*.h, the tile planner's invariants, the
Python mirror's configuration lowering, and the multi-process (gloo) timing
reduction used by bench.py for replicas."""
from __future__ import annotations

import os
import re
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    inc = os.path.join(ROOT, "include")
    for fn in sorted(os.listdir(inc)):
        if fn.endswith(".h"):
            src = open(os.path.join(inc, fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"\b(within_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(wb):
    import ctypes
    from within_b200 import _ffi
    lib = ctypes.CDLL(_ffi.LIB_PATH)
    decl = declared_functions()
    assert len(decl) >= 30
    missing = [n for n in decl if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(_ffi.exported_symbols()) == decl


def test_library_fails_loudly_without_gpu(wb):
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("a GPU is present")
    with pytest.raises(Exception):
        wb.Solver(np.asfortranarray(np.zeros((4, 2), np.uint32)))


def test_tile_planner_properties(tmp_path):
    exe = tmp_path / "plan_test"
    csrc = os.path.join(ROOT, "within_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", csrc, "-o", str(exe),
                    os.path.join(ROOT, "tests", "cpp", "plan_test.cpp"),
                    os.path.join(csrc, "host_design.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    assert "plan ok" in out


def test_locality_argsort(tmp_path):
    """The locality sort's stable argsort (one- and two-pass parallel forms
    and the counting sort) equals std::stable_sort (tests/cpp/argsort_test.cpp)."""
    exe = tmp_path / "argsort_test"
    csrc = os.path.join(ROOT, "within_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", csrc, "-o", str(exe),
                    os.path.join(ROOT, "tests", "cpp", "argsort_test.cpp"),
                    os.path.join(csrc, "host_design.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True, timeout=300).stdout
    assert "argsort ok 12" in out


def test_host_pool(tmp_path):
    """The set-up's host thread pool (host_pool.hpp): every item once, jobs
    posted from inside items and from several caller threads, the lowest
    failing index's exception rethrown, WITHIN_HOST_THREADS=1 serial on the
    caller (tests/cpp/pool_test.cpp)."""
    exe = tmp_path / "pool_test"
    csrc = os.path.join(ROOT, "within_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", csrc, "-o", str(exe),
                    os.path.join(ROOT, "tests", "cpp", "pool_test.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True, timeout=120).stdout
    assert "pool ok" in out


def test_segsweep_planner_and_warp_algorithm(tmp_path):
    """The warp-range segmented sweep (segsweep.cuh) executed lane by lane on
    the host over random multi-problem layouts planned by SSHostPlan::add:
    every segment emitted once with its exact sum, every position read once,
    every table index in range (tests/cpp/segsweep_test.cpp)."""
    exe = tmp_path / "segsweep_test"
    csrc = os.path.join(ROOT, "within_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", csrc, "-o", str(exe),
                    os.path.join(ROOT, "tests", "cpp", "segsweep_test.cpp"),
                    os.path.join(csrc, "host_design.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    assert "segsweep ok" in out


def test_schwarz_build_from_gpu_form_cross_tabs(tmp_path):
    """The additive-Schwarz build from cross-tabs in the GPU cross-tab's form
    (sorted keys, per-cell sums in observation order, CSR + CSC over raw level
    ids) gives the host-accumulated build's image bit for bit: unweighted,
    weighted with zero weights, slopes, unused levels, round factors; also
    when the cross-tabs arrive late, one pair at a time, through the per-pair
    futures the build waits on (tests/cpp/xtab_test.cpp)."""
    exe = tmp_path / "xtab_test"
    csrc = os.path.join(ROOT, "within_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", csrc, "-o", str(exe),
                    os.path.join(ROOT, "tests", "cpp", "xtab_test.cpp"),
                    os.path.join(csrc, "host_design.cpp"), os.path.join(csrc, "host_schwarz.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    assert "xtab ok 24" in out


def test_schwarz_round_schedule_and_index_ranges(tmp_path):
    """The round-parallel approximate-Cholesky schedule (no row of a round
    reads a row of the same round, forward or backward) and the index range of
    every array the Schwarz apply kernels gather through, on random designs
    (tests/cpp/schwarz_test.cpp)."""
    exe = tmp_path / "schwarz_test"
    csrc = os.path.join(ROOT, "within_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", csrc, "-o", str(exe),
                    os.path.join(ROOT, "tests", "cpp", "schwarz_test.cpp"),
                    os.path.join(csrc, "host_schwarz.cpp"), os.path.join(csrc, "host_design.cpp")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    assert "schwarz ok" in out


def test_dense_generalised_inverse(tmp_path):
    """The dense route's generalised inverse (LDL^T with a null pivot zeroed,
    host_schwarz.cpp dense_pinv) of connected and two-component Laplacians and
    of an SDD matrix (tests/cpp/pinv_test.cpp): symmetric, A G A = A, the
    inverse of the SDD matrix, and for the connected Laplacian the inverse
    grounded at the last vertex (natural order puts the null pivot there);
    relative to the largest entry, 1e-8."""
    import numpy as np
    exe = tmp_path / "pinv_test"
    csrc = os.path.join(ROOT, "within_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", csrc, "-o", str(exe),
                    os.path.join(ROOT, "tests", "cpp", "pinv_test.cpp"),
                    os.path.join(csrc, "host_schwarz.cpp"), os.path.join(csrc, "host_design.cpp")], check=True)
    lines = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines()
    assert lines[-1] == "pinv done"
    cases = 0
    for i in range(0, len(lines) - 1, 3):
        _, n, kind, size = lines[i].split()
        n = int(n)
        a = np.array(lines[i + 1].split(), float).reshape(n, n)
        g = np.array(lines[i + 2].split(), float).reshape(n, n)
        assert int(size) == n * n
        scale = np.max(np.abs(g))
        assert np.max(np.abs(g - g.T)) <= 1e-12 * scale
        assert np.max(np.abs(a @ g @ a - a)) <= 1e-8 * np.max(np.abs(a)), (n, kind)
        if kind == "2":
            ref = np.linalg.inv(a)
        elif kind == "0":
            ref = np.zeros_like(a)
            ref[:-1, :-1] = np.linalg.inv(a[:-1, :-1])
        else:
            ref = None
        if ref is not None:
            assert np.max(np.abs(g - ref)) <= 1e-8 * np.max(np.abs(ref)), (n, kind)
        cases += 1
    assert cases == 9


def test_config_lowering(wb):
    from within_b200 import _precond_config
    from within_b200.config import (AdditiveSchwarz, ApproxCholConfig, ApproxSchurConfig,
                                    LocalSolverConfig, ScalingConfig, Schur)
    assert _precond_config(None) is None
    assert _precond_config(wb.PreconditionerConfig.Off).kind == 0
    assert _precond_config(wb.PreconditionerConfig.Diagonal).kind == 2
    d = _precond_config(wb.PreconditionerConfig.Additive)
    assert (d.kind, d.dense_threshold, d.approx_chol_split, d.schur_split) == (1, 24, 2, 1)
    c = _precond_config(AdditiveSchwarz(local_solver=LocalSolverConfig(
        approx_chol=ApproxCholConfig(seed=3, split_merge=4),
        schur=Schur.approximate(ApproxSchurConfig(seed=5, split=2)), dense_threshold=7,
        scaling=ScalingConfig(tolerance=1e-6, max_sweeps=9, on_failure="error"))))
    assert (c.approx_chol_seed, c.approx_chol_split, c.schur_seed, c.schur_split) == (3, 4, 5, 2)
    assert (c.dense_threshold, c.scaling_tolerance, c.scaling_max_sweeps, c.scaling_error) == (7, 1e-6, 9, 1)
    assert _precond_config(AdditiveSchwarz(local_solver=LocalSolverConfig(schur=Schur.exact()))).schur_exact == 1
    with pytest.raises(ValueError):
        ApproxSchurConfig(split=0)
    with pytest.raises(TypeError):
        _precond_config("nope")


def test_layout_and_effect_validation(wb):
    lay = wb.CoefficientLayout([(0, 3, 1), (3, 4, 2)], 11)
    for i in range(11):
        assert lay.index(*lay.address(i)) == i
    with pytest.raises(IndexError):
        lay.index(1, 0, 2)
    with pytest.raises(IndexError):
        lay.address(11)
    with pytest.raises(ValueError):
        wb.Effect(np.zeros(4, np.uint32), False)
    with pytest.raises(ValueError):
        wb.Effect(np.zeros(4, np.uint32), True, [np.zeros(3)])
    with pytest.raises(TypeError):
        wb.Effect(np.zeros(4, np.float64), True)


def _replica_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t = bench.max_over_ranks(1.0 + rank, world)
    q.put((rank, t, bench.dist_env()))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks_gloo():
    import multiprocessing as mp
    import socket
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    q = ctx.Queue()
    procs = [ctx.Process(target=_replica_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.0, 2.0]
    assert [r[2][:2] for r in res] == [(0, 2), (1, 2)]


@pytest.mark.parametrize("budget", ["150", "0.001"])
def test_reference_arm_line(budget):
    """`bench.py --impl reference` (the oracle on the host's threads) honours
    --steps/--warmup and prints the reference line, with full-solve steps
    and, under a tiny time budget, bounded iteration samples."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--rows",
                          "20000", "--steps", "2", "--warmup", "2", "--ref-budget-s", budget],
                         cwd=root, capture_output=True, text=True, timeout=600, check=True).stdout
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 2
    assert line["value"] > 0 and line["unit"] == "solves/s" and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert ("per step one full solve" in line["cpu_baseline"]["sample"]) == (budget == "150")


def test_tuning_table_lookup():
    """The autotuner's table lookup (within_b200/autotune.py): nearest entry by
    weighted key distance, None beyond the distance limit or for an empty
    table; the design key of a worker/firm/year panel."""
    from within_b200 import autotune as A
    k = A.design_key(10_000_000, [1_000_000, 100_000, 20], False, False)
    assert k == [pytest.approx(23.2534966), 3.0, pytest.approx(19.9315686), pytest.approx(16.6096405), 0.0, 0.0]
    table = [{"key": A.design_key(2_000_000, [200_000, 20_000, 20], False, False), "tuning": {"fuse_rounds": 0}},
             {"key": A.design_key(100_000, [500, 200], False, False), "tuning": {"fuse_rounds": 1}}]
    assert A.lookup(k, table) == {"fuse_rounds": 0}
    assert A.lookup(A.design_key(120_000, [600, 150], False, False), table) == {"fuse_rounds": 1}
    assert A.lookup(A.design_key(1_000, [10], True, True), table) is None
    assert A.lookup(k, []) is None
