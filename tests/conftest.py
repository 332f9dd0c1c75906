"""Test configuration: import paths and the ``gpu`` marker.

``-m "not gpu"`` runs the oracle against the golden vectors, the host logic
and the C-ABI surface on any machine; ``-m gpu`` runs the parity tests proper
on a B200.
"""

from __future__ import annotations

import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for path in (ROOT, os.path.join(ROOT, "digital-fauxice_b200"), os.path.join(ROOT, "tests", "golden")):
    if path not in sys.path:
        sys.path.insert(0, path)

GOLDEN_PATH = os.path.join(ROOT, "tests", "golden", "reference_results.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built library")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def golden():
    with open(GOLDEN_PATH) as handle:
        return json.load(handle)
