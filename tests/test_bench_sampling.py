"""bench.py's CPU side: the oracle over the fixed root sample, the reference
arm's independence from the product library, and identical configs."""
import json
import os
import subprocess
import sys

import bench
import matrixgraph_b200 as mg
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_oracle_sample_counts_the_strided_positions():
    g = mg.rmat(13, 16, 0.57, 0.19, 0.19, seed=0, n_labels=4, label_kind="zipf", zipf_s=1.0,
                label_seed=1)
    names = list(bench.SHAPES)
    qs = [mg.query_walk(g, bench.SHAPES[s], seed=bench.SHAPE_SEED + i)
          for i, s in enumerate(names)]
    og = O.Graph.from_csr(g)
    oqs = [O.query_from_csr(q) for q in qs]
    saved = dict(bench.SAMPLE)
    try:
        bench.SAMPLE.update({s: (1 + i, 3 + i) for i, s in enumerate(names)})
        rows = bench.oracle_sample(og, oqs, names, 2)
    finally:
        bench.SAMPLE.clear()
        bench.SAMPLE.update(saved)
    for (name, b, s, nb, c, dt), oq in zip(rows, oqs):
        order = O.reference_order(oq)
        # the strided sample is the union of single-root counts at its positions
        want = sum(O.count(og, oq, order=order, root_range=(r, r + 1))["count"]
                   for r in range(b, nb, s))
        assert c == want, name
        assert dt >= 0.0


def test_reference_arm_loads_no_product_code_and_matches_config():
    """The reference arm builds its workload with the oracle's generator: the
    product package is never imported and libmg_subiso.so never mapped; its
    config equals the GPU arm's config for the same graph."""
    code = (
        "import sys, json, io, contextlib\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--scale', '12', '--steps', '1',"
        " '--warmup', '0']\n"
        "import bench\n"
        "buf = io.StringIO()\n"
        "with contextlib.redirect_stdout(buf):\n"
        "    bench.main()\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'line': json.loads(buf.getvalue()),"
        " 'pkg': 'matrixgraph_b200' in sys.modules, 'so': 'libmg_subiso' in maps}))\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert not out["pkg"] and not out["so"]
    line = out["line"]
    assert line["impl"] == "reference"
    g = mg.rmat(12, 16, 0.57, 0.19, 0.19, seed=0, n_labels=32, label_kind="zipf", zipf_s=1.0,
                label_seed=1)
    assert line["config"] == bench.config(12, g.n, g.m_out)
    assert set(line["sample_counts"]) == set(bench.SHAPES)
