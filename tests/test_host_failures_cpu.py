"""Host-side failure handling (no GPU): an allocation failure is injected into
the Python layer's workspace cache by replacing torch's allocator with a fake
that raises, and the cache logic is exercised with a fake that hands out CPU
tensors.  Nothing here touches a device."""
import torch

from tsm_benchmark_b200 import api

DEV = torch.device("cuda", 0)   # an explicit index: the cache never asks torch for the current device


def _clear(monkeypatch):
    monkeypatch.setattr(api, "_workspaces", {})


def test_workspace_allocation_failure_propagates_and_leaves_no_entry(monkeypatch):
    _clear(monkeypatch)

    def oom(*args, **kwargs):
        raise torch.OutOfMemoryError("injected: no device memory left")

    monkeypatch.setattr(torch, "zeros", oom)
    try:
        api.workspace(DEV, 1 << 22, 7)
    except torch.OutOfMemoryError as e:
        assert "injected" in str(e)
    else:
        raise AssertionError("the allocation failure was swallowed")
    assert api._workspaces == {}


def test_failed_growth_keeps_the_smaller_workspace(monkeypatch):
    _clear(monkeypatch)
    real_zeros = torch.zeros
    made = []

    def fake(n, dtype=None, device=None):
        made.append(n)
        return real_zeros(n, dtype=dtype)

    monkeypatch.setattr(torch, "zeros", fake)
    small = api.workspace(DEV, 1000, 7)
    assert small.numel() == 1 << 20 and made == [1 << 20]   # at least 1 MiB, zero-filled
    assert not small.any()

    def oom(*args, **kwargs):
        raise torch.OutOfMemoryError("injected")

    monkeypatch.setattr(torch, "zeros", oom)
    try:
        api.workspace(DEV, 1 << 24, 7)
    except torch.OutOfMemoryError:
        pass
    else:
        raise AssertionError("the allocation failure was swallowed")
    # the entry still holds the earlier workspace, which serves requests it fits
    monkeypatch.setattr(torch, "zeros", fake)
    assert api.workspace(DEV, 1 << 20, 7) is small


def test_workspace_cache_per_device_and_stream(monkeypatch):
    _clear(monkeypatch)
    real_zeros = torch.zeros
    made = []

    def fake(n, dtype=None, device=None):
        made.append((n, device))
        return real_zeros(n, dtype=dtype)

    monkeypatch.setattr(torch, "zeros", fake)
    a = api.workspace(DEV, 4096, 1)
    assert api.workspace(DEV, 100, 1) is a                     # reused on the same stream
    b = api.workspace(DEV, 4096, 2)                              # another stream: its own
    assert b is not a
    c = api.workspace(torch.device("cuda", 1), 4096, 1)          # another device: its own
    assert c is not a and c is not b
    grown = api.workspace(DEV, (1 << 20) + 1, 1)                 # larger than held: replaced
    assert grown.numel() == (1 << 20) + 1 and api.workspace(DEV, 10, 1) is grown
    assert [n for n, _ in made] == [1 << 20, 1 << 20, 1 << 20, (1 << 20) + 1]
    assert all(d == DEV or d == torch.device("cuda", 1) for _, d in made)
