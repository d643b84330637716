"""smoke() of the repository's entry module: one small blastp --sensitive
search on cuda:0 through the library, checked HSP for HSP against the oracle.
"""
import importlib.util
import os

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_entry_smoke():
    spec = importlib.util.spec_from_file_location("repo_entry", os.path.join(ROOT, "__graft_entry__.py"))
    entry = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(entry)
    entry.smoke()  # raises when the GPU's HSPs differ from the oracle's or there are none
