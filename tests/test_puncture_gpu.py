"""Permutation::permute / dePermute on the GPU (fecl_permute): numpy's gather and
scatter semantics for every element type, zero-filled punctured positions, the
reference's last-writer rule for repeated indices; and a punctured rate-1/2 LTE
chain (encode, puncture, channel, depuncture, decode) run entirely on the GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.float16, np.uint8])
def test_permute_and_depermute_semantics(dtype):
    import torch
    import fecl_b200 as F
    rng = np.random.default_rng(70)
    n_in, n_out, blocks = 1000, 600, 7
    seq = np.sort(rng.choice(n_in, n_out, replace=False)).astype(np.uint32)
    rng.shuffle(seq)
    p = F.Permutation(seq, n_in)
    x = (rng.integers(0, 200, size=blocks * n_in)).astype(dtype)
    y = p.permute(x)
    assert np.array_equal(y, x.reshape(blocks, n_in)[:, seq].ravel())
    z = p.dePermute(y)
    ref = np.zeros((blocks, n_in), dtype)
    ref[:, seq] = y.reshape(blocks, n_out)
    assert np.array_equal(z, ref.ravel())
    # device tensors stay on the device
    t = torch.from_numpy(x).cuda()
    assert torch.equal(p.permute(t).cpu(), torch.from_numpy(y))


def test_repeated_indices_last_writer_wins():
    import fecl_b200 as F
    seq = np.array([3, 1, 3, 0], np.uint32)
    p = F.Permutation(seq, 5)
    out = p.dePermute(np.array([10, 11, 12, 13], np.float32))
    assert np.array_equal(out, np.array([13, 11, 0, 12, 0], np.float32))


def test_punctured_lte_chain_on_the_gpu():
    import torch
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    K = 1024
    code = F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(8))
    perm = code.puncturing(F.Turbo.PunctureOptions().mask([[1], [1, 0], [0, 1]]))
    n = 32
    rate = K / perm.outputSize()
    assert abs(rate - 0.5) < 0.01
    msg = torch.randint(0, 2, (n * K,), dtype=torch.uint8, device="cuda")
    tx = perm.permute(code.encode(msg))
    rx = ch.awgn_llr_device(tx, 3.0, rate, 71)
    llr = perm.dePermute(rx)
    assert llr.numel() == n * code.paritySize()
    assert torch.equal(code.decode(llr), msg)
