"""The multi-rank launch path of bench.py on CPU (gloo, world size 2): ranks
agree on the max-over-ranks time, and only rank 0 prints its JSON line.  The
GEMM has no exchange step, so N > 1 runs independent replicas."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_two_ranks_gloo():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", "29631", os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--size", "256", "--slices", "4", "--steps", "1",
           "--warmup", "0", "--cpu-sample", "64"]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="2")
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["e2e"]["h2d_bytes_per_step"] == 0 and rec["cpu_baseline"]["kind"] == "reference"


def _max_worker(rank, ws, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    sys.path.insert(0, ROOT)
    import bench
    q.put((rank, bench.dist_max(float(rank + 1) * 1.5, ws)))
    bench.barrier(ws)
    dist.destroy_process_group()


def test_dist_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_max_worker, args=(r, 2, 29632, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == {0: 3.0, 1: 3.0}


def test_reference_arm_loads_only_the_checkers():
    """The reference arm runs the reference's own code only: its inputs come
    from the reference's generator and its steps from the reference's kernel
    source, both in oracle/_ref; this repository's library is never loaded."""
    import pytest
    sys.path.insert(0, ROOT)
    from oracle import ref_available
    if not ref_available():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    code = (
        "import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--size', '256', '--slices', '4',"
        " '--steps', '1', '--warmup', '0', '--cpu-sample', '64']\n"
        "import runpy; runpy.run_path('bench.py', run_name='__main__')\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('LOADED', json.dumps({'pkg': 'ozablas_b200' in sys.modules, 'lib': 'liboza_b200' in maps,"
        " 'ref': 'libozaref_cpu' in maps}))\n")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="2")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    loaded = json.loads(out.stdout.split("LOADED", 1)[1])
    assert loaded == {"pkg": False, "lib": False, "ref": True}
