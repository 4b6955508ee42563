"""Shared fixtures: generated problems (in memory and as reference-format files)."""
import os
import sys
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


_CACHE = {}


def make_problem(name, **kw):
    """JProblem for a named workload (cached per session)."""
    from nushellx_b200.gen.space import WORKLOADS
    from nushellx_b200.gen.problem import JProblem
    key = (name, tuple(sorted(kw.items())))
    if key not in _CACHE:
        _CACHE[key] = JProblem.from_workload(WORKLOADS[name], **kw)
    return _CACHE[key]


def custom_problem(space_name, nprot, nneut, J2, parity, seed):
    from nushellx_b200.gen import space as S
    from nushellx_b200.gen.problem import JProblem
    key = ("custom", space_name, nprot, nneut, J2, parity, seed)
    if key not in _CACHE:
        sp = getattr(S, space_name)
        w = S.Workload("custom", sp, nprot, nneut, J2, parity, seed)
        _CACHE[key] = JProblem.from_workload(w)
    return _CACHE[key]


@pytest.fixture(scope="session")
def files_dir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("nsx_files"))


def write_files(P, d, tag):
    from nushellx_b200.gen.writer import write_problem
    key = ("files", id(P), d, tag)
    if key not in _CACHE:
        _CACHE[key] = write_problem(P, d, tag)
    return _CACHE[key]


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
