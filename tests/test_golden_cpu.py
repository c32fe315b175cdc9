"""The oracle (through the product's own front end) against the committed golden fixtures,
which were produced by the reference itself (tests/golden/make_golden.py)."""
import os
import subprocess

import pytest

import ffi
import golden_cases


@pytest.fixture(scope="module", autouse=True)
def _built():
    subprocess.run(["make", "-s", "-C", ffi.ORACLE_DIR, "storm-oracle-nucleotide", "storm-oracle-color"],
                   check=True)


@pytest.mark.parametrize("name", sorted(golden_cases.meta()))
def test_oracle_matches_golden(name, tmp_path):
    exe = lambda mode: os.path.join(ffi.ORACLE_DIR, "storm-oracle-color" if mode == "colour"
                                    else "storm-oracle-nucleotide")
    assert golden_cases.check_case(name, str(tmp_path), exe) > 0
