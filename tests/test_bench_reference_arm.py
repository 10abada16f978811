"""The bench's reference arm (`bench.py --impl reference`) runs on the host
alone: one small scene through the reference's own CPU build must print the
contract's JSON line."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_its_line():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libccref_f32.so")):
        pytest.skip("the reference's CPU build is absent (make -C oracle ref)")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1", "--n", "20000"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1])
    assert line["impl"] == "reference" and line["metric"] == "bodies/s" and line["value"] > 0
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "reference"
    assert line["result"]["pairs"] > 0
    assert set(line["stages_ms_mean"]) == {"generate_aabb", "detect_possible_collisions", "do_narrowphase"}
    # the process that timed the reference's CPU build mapped none of this
    # repository's GPU code (read from its own /proc/self/maps)
    libs = line["native_libraries"]
    assert "oracle/_ref/libccref_f32.so" in libs
    assert not any("libcollide_b200" in p for p in libs), libs


def test_both_arms_print_the_same_config():
    # the driver compares the two arms' `config` objects
    sys.path.insert(0, ROOT)
    import bench
    assert bench.workload_config(1 << 20, 1)["workload"] == bench.WORKLOAD
    assert bench.workload_config(1 << 20, 1) == bench.workload_config(1 << 20, 1)


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_under_torchrun_over_gloo():
    # the launch the driver uses for N > 1, on the host: rank 0 prints one line,
    # rank 1 leaves without work, both exit 0
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libccref_f32.so")):
        pytest.skip("the reference's CPU build is absent (make -C oracle ref)")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "1", "--bodies", "20000"]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1 and json.loads(lines[0])["n_gpus"] == 2


_MAX_OVER_RANKS = r'''
import os, sys
sys.path.insert(0, sys.argv[1])
import bench
world, rank, _ = bench.dist_setup(2)
bench.dist_barrier(world)
v = bench.dist_max(10.0 + rank, world)
assert world == 2 and v == 11.0, (world, v)  # every rank sees the maximum
if rank == 0:
    print("max", v, flush=True)
'''


def test_max_over_ranks_over_gloo(tmp_path):
    script = tmp_path / "max_over_ranks.py"
    script.write_text(_MAX_OVER_RANKS)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), str(script), ROOT]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    assert [ln for ln in out.stdout.splitlines() if ln.startswith("max")] == ["max 11.0"]
