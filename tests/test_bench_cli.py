"""bench.py on the CPU: every global name its functions use is defined (a
missing helper would otherwise surface only on the GPU box), the kernel
source digests print, and the reference arm (the reference's CPU presolver)
runs on the 2,000 x 5,000 workload and prints one well-formed JSON line."""
import builtins
import json
import os
import subprocess
import sys
import symtable

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "bench.py")


def _undefined_globals(path):
    src = open(path).read()
    top = symtable.symtable(src, path, "exec")
    defined = {s.get_name() for s in top.get_symbols() if s.is_assigned() or s.is_imported()}
    defined |= set(dir(builtins))
    missing = []

    def walk(table):
        for sym in table.get_symbols():
            if sym.is_referenced() and sym.is_global() and sym.get_name() not in defined:
                missing.append((table.get_name(), sym.get_name()))
        for child in table.get_children():
            walk(child)

    for child in top.get_children():
        walk(child)
    return missing


def test_bench_uses_no_undefined_global():
    assert _undefined_globals(BENCH) == []


def test_source_digests_print():
    r = subprocess.run([sys.executable, BENCH, "--source-digests"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "candidates_entries" in r.stdout


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "pslp_driver")),
                    reason="reference CPU presolver not built")
def test_reference_arm_small_workload():
    r = subprocess.run([sys.executable, BENCH, "--impl", "reference", "--steps", "2", "--warmup", "1",
                        "--workload", "small"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "ms" and line["steps"] == 2
    assert line["cpu_baseline"]["kind"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
