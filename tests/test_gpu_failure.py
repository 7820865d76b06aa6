"""Failure detection without a GPU fault: every wait inside the tensor-core
selector kernel is bounded.  Here a wait is made to run out (the kernel's
weight producer withheld, so the weights it waits for never arrive): the
kernel must return an error status to the host within its limit, and the
device must stay usable -- a normal run of the same kernel and a whole
compression afterwards succeed and are exact."""
import time

import numpy as np
import pytest
import torch

import bzip2gpu_b200 as B
import bzip2gpu_b200.selector as S
import oracle

pytestmark = pytest.mark.gpu


def _syms(n=30000, seed=5):
    rng = np.random.default_rng(seed)
    return torch.from_numpy(rng.integers(0, 40, n).astype(np.int16)).cuda()


def test_withheld_producer_times_out_and_device_recovers(torch_cuda):
    d_syms = _syms()
    d_P = torch.from_numpy(S.load()).cuda()
    t0 = time.perf_counter()
    with pytest.raises(B.Bz2gError) as e:
        B.selector_wait_check(d_syms, d_P, 200_000, withhold_weights=True)  # 200 us
    elapsed = time.perf_counter() - t0
    assert e.value.code == B.ERR_TIMEOUT
    assert "bounded wait ran out" in str(e.value)
    assert elapsed < 30, elapsed  # the kernel returned on its own limit
    # the context is intact: the same kernel with its producer meets every wait
    B.selector_wait_check(d_syms, d_P, 2_000_000_000, withhold_weights=False)
    # ... and agrees with the entry point that runs it for real
    lg, sel = B.selector_logits(d_syms, d_P)
    assert sel.numel() == (d_syms.numel() + 49) // 50
    data = oracle.large_stream(1 << 20)
    assert B.compress(data, 9) == oracle.compress(data, 9, threads=4)


def test_wait_limit_must_be_positive(torch_cuda):
    with pytest.raises(B.Bz2gError) as e:
        B.selector_wait_check(_syms(1000), torch.zeros(B.SELECTOR_PARAMS, device="cuda"), 0,
                              False)
    assert e.value.code == 2
