"""Shared test configuration: the `gpu` marker and the import path.

Tests marked `gpu` need a CUDA device and the built library; everything else
runs on the CPU (the oracle, host logic, the C-ABI's exported symbols).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built gargantua_b200 library")
    config.addinivalue_line("markers", "slow: long CPU oracle runs")


GOLDEN_DIR = os.path.join(TESTS, "golden", "goldens")


def load_golden(name: str) -> dict:
    import json

    with open(os.path.join(GOLDEN_DIR, name + ".json")) as fh:
        return json.load(fh)


def golden_passes(golden: dict, measured: float) -> bool:
    """Golden.passes (Sources/Oracle/Golden.swift:45-51)."""
    kind = golden["kind"]
    if kind == "relative":
        return abs(measured - golden["expected"]) / abs(golden["expected"]) <= golden["tolerance"]
    if kind == "absolute":
        return abs(measured - golden["expected"]) <= golden["tolerance"]
    return measured == golden["expected"]
