"""Test configuration: the `gpu` marker, import paths and shared fixtures.

Tests marked `gpu` need a B200 and the built library; everything else runs on the CPU
(oracle, golden fixtures, host logic, library symbols).
"""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "sbd-pub_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def golden_cases():
    return json.load(open(os.path.join(GOLDEN, "cases.json")))


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def golden_problem(name):
    """The case's Problem (strings from the fixture; integrals regenerated or read)."""
    from sbd_tpb import Problem
    meta = golden_cases()[name]
    g = load_golden(name)
    h1, eri, core = g["h1"], g["eri"], float(g["core"][0])
    nelec = int(bin(int(g["astr"][0])).count("1") + bin(int(g["bstr"][0])).count("1"))
    return Problem(norb=meta["norb"], nelec=nelec, core=core, h1=h1, eri_packed=eri,
                   astr=g["astr"], bstr=g["bstr"]), g, meta


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    pyoracle.lib()
    return pyoracle
