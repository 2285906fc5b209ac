"""The capacity path (after the reference's residency probe,
tests/cuda_capacity.cu:48-157): a population generated directly in device
memory -- random 32-bit words, every one a valid instruction
(src/ISA.h:106-138) -- evaluated where it lies with
galop_evaluate_csr_device.  Its fitness must equal the host-pointer call's on
the same words bit for bit, and the evaluator's own device memory per
program must stay within the footprint the capacity measurement assumes."""
from __future__ import annotations

import numpy as np
import pytest

import galop_b200 as g
from conftest import bits

pytestmark = pytest.mark.gpu


def test_device_generated_population_matches_host_call(native):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    P, L, D = 1 << 20, 30, 32
    rng = np.random.default_rng(1234)
    x = rng.uniform(-1, 1, (D, 1)).astype(np.float32)
    y = (x[:, 0] ** 3 + x[:, 0] ** 2 + x[:, 0]).astype(np.float32)
    gen = torch.Generator(device=dev)
    gen.manual_seed(7)
    w = torch.randint(-2**31, 2**31 - 1, (P * L,), dtype=torch.int32, device=dev, generator=gen)
    off = torch.arange(P + 1, dtype=torch.int64, device=dev) * L
    fit = torch.empty(P, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    with g.Evaluator(num_registers=8) as ev:
        ev.set_dataset(g.Dataset(x, y))
        free0 = torch.cuda.mem_get_info(dev)[0]
        ev.evaluate_csr_device(w.data_ptr(), off.data_ptr(), P, P * L, fit.data_ptr())
        st = ev.stats
        used = free0 - torch.cuda.mem_get_info(dev)[0]
        dev_fit = fit.cpu().numpy()
        host_fit = ev.evaluate_csr(w.cpu().numpy().view(np.uint32), off.cpu().numpy())
    assert st.raw_instructions == P * L and 0 < st.eff_instructions < 0.3 * P * L
    assert np.array_equal(bits(dev_fit), bits(host_fit))
    # the evaluator's buffers for this population (micro-ops sized for the
    # raw words on the asynchronous path, offsets, order, dedup keys,
    # partial sums): well under 1 KB per 30-word program
    assert used / P < 1024, used / P
