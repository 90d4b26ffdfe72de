"""CPU: a C translation unit includes include/rtt_spgemm.h, links
librtt_spgemm.so and runs (no GPU call); its SMatrix layout (sizeof and the
offset of every field) equals the reference's SMatrix (src/common.h:50-72),
printed by oracle/_ref/ref_layout, which is compiled from the reference's own
header."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

import rtt_spgemm as R

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "c_abi" / "abi_layout.c"
REF_LAYOUT = ROOT / "oracle" / "_ref" / "ref_layout"


def _layout(text: str) -> dict:
    out = {}
    for line in text.splitlines():
        k, _, v = line.partition(" ")
        out[k] = v
    return out


@pytest.fixture(scope="module")
def c_caller(tmp_path_factory):
    cc = shutil.which("gcc") or "/usr/bin/gcc"
    exe = tmp_path_factory.mktemp("c_abi") / "abi_layout"
    lib = Path(R.LIB_PATH)
    subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(SRC),
                    "-o", str(exe), "-L", str(lib.parent), "-lrtt_spgemm",
                    "-Wl,-rpath," + str(lib.parent)], check=True)
    res = subprocess.run([str(exe)], check=True, capture_output=True, text=True)
    return _layout(res.stdout)


def test_c_caller_compiles_links_and_runs(c_caller):
    assert "sm_100a" in c_caller["version"]
    assert c_caller["status2"] == "invalid CSR"


def test_smatrix_offsets_match_the_reference_header(c_caller):
    if not REF_LAYOUT.exists():
        pytest.skip("oracle/_ref/ref_layout not built (needs the reference checkout)")
    ref = _layout(subprocess.run([str(REF_LAYOUT)], check=True, capture_output=True,
                                 text=True).stdout)
    fields = [k for k in ref if k != "sizeof"]
    assert len(fields) == 20
    for k in ["sizeof"] + fields:
        assert c_caller[k] == ref[k], f"{k}: {c_caller[k]} != reference {ref[k]}"
