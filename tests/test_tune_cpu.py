"""The batched form's autotuner on the host: its cache keys, its choice among measured candidates and its cache text
are deterministic, and a batch refuses to run without a GPU instead of falling back."""
import ctypes

import pytest

from conftest import cuda_ok
from nereus_cfd_b200 import build, capi, serving


@pytest.fixture(scope="module")
def lib():
    build.build()
    return capi.load()


def key(lib, *args):
    buf = ctypes.create_string_buffer(128)
    n = lib.nereus_b200_tune_key(*args, buf, 128)
    assert n == len(buf.value)
    return buf.value.decode()


def choose(lib, times, fallback=0):
    arr = (ctypes.c_double * len(times))(*times)
    return lib.nereus_b200_tune_choose(len(times), arr, fallback)


def test_keys_name_grid_level_kind_and_capacity(lib):
    k = key(lib, 130, 130, 130, 0, 1, 64)
    assert k == "split 130x130x130 L0 half B64"
    assert key(lib, 130, 130, 130, 0, 1, 64) == k
    others = {key(lib, 130, 130, 130, 1, 1, 64), key(lib, 130, 130, 130, 0, 2, 64), key(lib, 130, 130, 130, 0, 1, 8),
              key(lib, 66, 66, 66, 0, 1, 64), key(lib, 130, 130, 66, 0, 1, 64)}
    assert k not in others and len(others) == 5
    assert [key(lib, 10, 10, 10, 0, kind, 1).split()[3] for kind in range(5)] == capi.BATCH_KINDS
    assert lib.nereus_b200_tune_key(10, 10, 10, 0, 5, 1, ctypes.create_string_buffer(64), 64) == capi.NB_BAD_INPUT


def test_choice_rules(lib):
    # the fastest
    assert choose(lib, [10.0, 8.0, 9.0]) == 1
    # the fallback when within 3% of the fastest
    assert choose(lib, [10.0, 9.8, 9.9], fallback=0) == 0
    assert choose(lib, [10.0, 9.6, 9.9], fallback=0) == 1
    # ties within 0.5% go to the earlier candidate, whatever the order of the measurement noise
    assert choose(lib, [10.0, 8.0, 7.99, 7.97], fallback=0) == 1
    # unusable times are skipped; with none the fallback
    assert choose(lib, [float("nan"), 0.0, 5.0], fallback=0) == 2
    assert choose(lib, [float("nan"), -1.0], fallback=1) == 1
    # the same inputs, the same answer
    ts = [12.5, 11.1, 11.0, 13.0, 11.05]
    assert len({choose(lib, ts, 3) for _ in range(20)}) == 1


def test_cache_text_round_trip(lib):
    lib.nereus_b200_tune_cache_clear()
    assert serving.tune_cache_dump() == ""
    text = "split 130x130x130 L0 half B64|4|0|812.500\nsplit 66x66x66 L1 restrict B64|2|1|40.250\n"
    assert serving.tune_cache_load(text) == 2
    assert serving.tune_cache_dump() == "".join(sorted(text.splitlines(True)))
    # a malformed text adds nothing
    assert lib.nereus_b200_tune_cache_load(b"split 1x1x1 L0 half B1|0|0|1.0\n") == capi.NB_BAD_INPUT
    assert lib.nereus_b200_tune_cache_load(b"no separator\n") == capi.NB_BAD_INPUT
    assert serving.tune_cache_dump().count("\n") == 2
    lib.nereus_b200_tune_cache_clear()
    assert serving.tune_cache_dump() == ""


def test_batch_checks_capacity_and_needs_a_device(lib):
    h = ctypes.c_void_p()
    assert lib.nereus_b200_batch_create(ctypes.byref(h), None, 0) == capi.NB_BAD_INPUT
    assert lib.nereus_b200_batch_create(ctypes.byref(h), None, 1025) == capi.NB_BAD_INPUT
    assert lib.nereus_b200_batch_project_device(None, 1, None, None) == capi.NB_BAD_INPUT
    if not cuda_ok():
        assert lib.nereus_b200_batch_create(ctypes.byref(h), None, 4) == capi.NB_NO_DEVICE
        assert not h
