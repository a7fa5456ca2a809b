"""The C ABI library and the drop-in programs, without a GPU.

Loads libcmfw.so, checks that it exports every function include/cmfw.h
declares, and exercises the host-only entry points (descriptors, input
records, the mt19937_64 stream) and the programs' argument handling, which
the reference performs before touching the device.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import cmfw
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cmfw.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cmfw_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    declared = header_functions()
    assert declared, "no declarations parsed"
    lib = cmfw.lib()
    missing = [f for f in declared if not hasattr(lib, f)]
    assert not missing, missing
    assert sorted(cmfw.EXPORTS) == declared


def test_version_string():
    assert "sm_100a" in cmfw.version()


@pytest.mark.parametrize("p,q,z,rank", [(3, 2, 0.5, 3), (3, 2, 1.0, 2), (4, 3, 1.0, 3), (5, 4, 0.5, 5),
                                        (6, 5, 1.0, 5), (6, 5, 0.5, 6), (8, 7, 1.0, 7), (8, 7, 0.5, 8),
                                        (2, 4, 1.0, 5), (5, 1, 1.0, 5)])
def test_rank_rule(p, q, z, rank):
    # make_cmf_desc (cmf_pfq.cuh:50-61)
    d = cmfw.make_desc(p, q, z)
    assert (d.p, d.q, d.naxes, d.rank) == (p, q, p + q, rank)
    assert oracle.ffi._oracle().orc_make_desc  # the oracle states the same rule
    cmfw.check_desc(d)


@pytest.mark.parametrize("p,q,z", [(9, 2, 0.5), (3, 8, 0.5), (0, 2, 0.5), (1, 0, 1.0)])
def test_unsupported_descriptors_rejected(p, q, z):
    with pytest.raises(cmfw.CmfwError):
        cmfw.check_desc(cmfw.make_desc(p, q, z))


def test_nonfinite_z_rejected():
    d = cmfw.make_desc(3, 2, 0.5)
    d.z = float("nan")
    with pytest.raises(cmfw.CmfwError, match="EINVAL"):
        cmfw.check_desc(d)


@pytest.mark.parametrize("p,q", [(3, 2), (4, 3), (5, 4), (6, 5), (8, 7)])
@pytest.mark.parametrize("mode,zeta", [(0, False), (0, True), (1, False), (1, True)])
def test_reference_inputs_match_oracle(p, q, mode, zeta):
    a = cmfw.reference_inputs(p, q, 999, mode, zeta)
    b = oracle.make_inputs(p, q, 999, mode, zeta)
    assert a.tobytes() == b.tobytes()


def test_reference_inputs_edge_sizes():
    assert len(cmfw.reference_inputs(3, 2, 0, 0, False)) == 0
    one = cmfw.reference_inputs(3, 2, 1, 1, False)
    assert one.tobytes() == oracle.make_inputs(3, 2, 1, 1, False).tobytes()


def test_mt64_known_answer():
    assert int(cmfw.mt64(5489, 10000)[-1]) == 9981545732273789042
    np.testing.assert_array_equal(cmfw.mt64(42, 100), oracle.mt64_stream(42, 100))


def test_workload_generators_deterministic():
    import cmfw.workloads as wl
    a = wl.zeta_directions(6, 5, 300, 7)
    b = wl.zeta_directions(6, 5, 300, 7)
    assert a.tobytes() == b.tobytes()
    d = a["dir"][:, :11]
    assert d.min() >= 0 and d.max() <= 3 and (np.abs(d).sum(1) > 0).all()
    assert (a["start"][:, :6] == 1).all() and (a["start"][:, 6:11] == 2).all()
    c = wl.zeta_directions(8, 7, 200, 9, lo=0, hi=2, offset=1)["dir"][:, :15]
    assert c.min() >= 1 and c.max() <= 3
    s = wl.limit_starts(3, 2, 500, 3)
    assert s["start"][:, :5].min() >= 1 and s["start"][:, :5].max() <= 10
    assert (s["dir"][:, :5] == 1).all()


def _cli(variant, *args):
    exe = os.path.join(cmfw.BIN_DIR, f"cmf_walk_{variant}")
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=60)


@pytest.mark.parametrize("variant", ["f64", "df64", "rns"])
def test_cli_rejects_unknown_flag(variant):
    r = _cli(variant, "--frobnicate")
    assert r.returncode == 1
    assert ("Unknown arg: --frobnicate" if variant == "f64" else "Unknown: --frobnicate") in r.stderr


def test_cli_missing_value_exits_1():
    r = _cli("f64", "--N")
    assert r.returncode == 1 and "Missing value after --N" in r.stderr
    assert _cli("df64", "--h").returncode == 1


def test_cli_bad_cmf_type():
    r = _cli("f64", "--cmf", "abc")
    assert r.returncode == 1 and "Invalid CMF type: abc" in r.stderr
    assert _cli("rns", "--cmf", "xFy").returncode == 1


def test_cli_n_primes_only_for_rns():
    assert _cli("f64", "--n-primes", "8").returncode == 1
    assert _cli("df64", "--n-primes", "8").returncode == 1
