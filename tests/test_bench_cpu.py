"""The benchmark's host-side pieces, without a GPU: the reference arm loads
nothing of the product package and prints the ours-arm's config; the bytes
model; the synthetic workloads' shapes and seeds."""
import json
import os
import subprocess
import sys

import numpy as np

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_loads_nothing_of_the_product():
    """`--impl reference` times the oracle on the host: its line carries the
    same config keys as the ours-arm's, and the process never imports the
    product package."""
    code = (
        "import runpy, sys\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0',\n"
        "            '--points', '20000', '--queries', '20000']\n"
        "try:\n"
        "    runpy.run_path('bench.py', run_name='__main__')\n"
        "except SystemExit:\n"
        "    pass\n"
        "print('PRODUCT_LOADED', any(m == 'kiddo_b200' or m.startswith('kiddo_b200.')\n"
        "                            for m in sys.modules))\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["config"] == bench.config_for("c2_knn16", 20000, 20000, 1)
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert "PRODUCT_LOADED False" in r.stdout


def test_bytes_per_query_model():
    # 10 queries that visited 100 stems, 20 leaves and 300 points in total:
    # query 12 B + 10 stems x 4 B + 30 points x 16 B + 16 entries x 8 B + 4 B
    b = bench.bytes_per_query((100, 20, 300), 10, 4, 16)
    assert b == 12 + 40 + 480 + 128 + 4
    # f64, one result, no count
    assert bench.bytes_per_query((10, 1, 20), 1, 8, 1) == 24 + 80 + 20 * 28 + 12


def test_workloads_are_seeded_and_shaped():
    P1, Q1 = bench.make_data("c2_knn16", 0, 5000, 3000)
    P2, Q2 = bench.make_data("c2_knn16", 0, 5000, 3000)
    assert P1.shape == (5000, 3) and Q1.shape == (3000, 3) and P1.dtype == np.float32
    assert np.array_equal(P1, P2) and np.array_equal(Q1, Q2)
    _, Q3 = bench.make_data("c2_knn16", 1, 5000, 3000)  # another rank: other queries
    assert not np.array_equal(Q1, Q3)
    P, Q = bench.make_data("c5_periodic", 0, 4000, 4000)
    assert P.dtype == np.float64 and P is Q  # every particle queries
    assert (P >= 0).all() and (P < 1).all()
    P, Q = bench.make_data("c1_nn1", 0, 1000, 2000)
    assert P.dtype == np.float64 and Q.shape == (2000, 3)


def test_kernel_names_follow_the_engine():
    assert bench.kernel_name("nearest_n", None) == "k_tfixed<nearest_n>"
    assert bench.kernel_name("nearest_n", "coop") == "k_tnn_coop"
    assert bench.kernel_name("approx", "warp") == "k_fixed<approx>"
    assert bench.kernel_name("periodic_nearest_n_within", None).startswith("k_tnn_coop")
