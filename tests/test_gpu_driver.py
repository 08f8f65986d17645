"""pava_bench, main.cpp's CVR / CSR5 benchmark loop over the C ABI: it runs, prints the
reference's Performance lines and passes the reference's 1 % check."""
import json
import os
import re
import subprocess

import pytest

from pava_b200 import build as B

pytestmark = pytest.mark.gpu

PERF = re.compile(r"^ Performance (\S+) (CVR|CSR5) (\d+) (-?[0-9.]+) (-?[0-9.]+) $", re.M)


def _run(*args):
    exe = B.build_driver()
    r = subprocess.run([exe, *args], capture_output=True, text=True, timeout=600)
    return r.returncode, r.stdout + r.stderr


def test_driver_laplace_c1(cuda):
    rc, out = _run("--laplace", "512", "200")
    assert rc == 0, out
    lines = PERF.findall(out)
    assert [l[1] for l in lines] == ["CVR", "CSR5"], out
    for name, fmt, sms, conv, exe in lines:
        assert name == "laplace_512" and int(sms) > 0 and float(conv) > 0 and float(exe) > 0
    assert "CVR status 0, rows off by more than 1%: 0" in out
    assert "CSR5 status 0, rows off by more than 1%: 0" in out
    # one machine-readable record per section beside the Performance line
    recs = [json.loads(l) for l in out.splitlines() if l.startswith('{"record": "pava_bench"')]
    assert [r["section"] for r in recs] == ["CVR", "CSR5"]
    for r in recs:
        assert r["status"] == 0 and r["matrix"] == "laplace_512" and r["nnz"] == 1_308_672
        assert r["GBps"] > 0 and 0 < r["roofline_frac"] < 2 and r["max_rel_err"] <= 1e-12
        assert r["rows_off_1pct"] == 0 and r["iterations"] == 200 and r["convert_s"] > 0
    assert recs[0]["steps"] in (32, 64, 128) and recs[1]["sigma"] == 16


def test_driver_mtx_and_small_cvr_guard(cuda, tmp_path):
    from pava_b200 import matrices as M
    A = M.powerlaw(3000, mean=8.0, seed=9)   # below main.cpp's 4096 guard: CVR skipped
    path = os.path.join(tmp_path, "small.mtx")
    M.write_mtx(path, A)
    rc, out = _run(path, "5")
    assert rc == 0, out
    lines = PERF.findall(out)
    assert lines[0][1] == "CVR" and float(lines[0][3]) == -1.0   # skipped, as in main.cpp
    assert lines[1][1] == "CSR5" and float(lines[1][4]) > 0


def test_driver_sell_section(cuda, tmp_path):
    """--sell adds a SELL section: on the Laplacian a Performance line and a record passing the
    same checks; on a power-law matrix one line saying why the form refuses it."""
    rc, out = _run("--laplace", "512", "50", "--sell")
    assert rc == 0, out
    assert "SELL status 0, rows off by more than 1%: 0" in out
    assert re.search(r"^ Performance laplace_512 SELL (\d+) ([0-9.]+) ([0-9.]+) $", out, re.M), out
    recs = [json.loads(l) for l in out.splitlines() if l.startswith('{"record": "pava_bench"')]
    assert [r["section"] for r in recs] == ["CVR", "CSR5", "SELL"]
    assert recs[2]["max_rel_err"] <= 1e-12 and recs[2]["rows_off_1pct"] == 0
    from pava_b200 import matrices as M
    A = M.powerlaw(8000, mean=8.0, seed=11)
    assert not M.sell_accepts(A)
    path = os.path.join(tmp_path, "pl.mtx")
    M.write_mtx(path, A)
    rc, out = _run(path, "5", "--sell")
    assert rc == 0, out
    assert "SELL refuses the matrix: SELL: padding" in out
