"""The radiance codec's device forms (a CUDA lane whose sums stay in GPU memory) against
the host codec: the same payload bytes from device f64 sums as the host encoder makes
from their f32 rounding, and the device valid-sample add bit-identical to the host's."""
import numpy as np
import pytest

from indicatrix_b200 import radiance as rad, workloads
from indicatrix_b200.radiance import PayloadDecoder, PayloadEncoder, PayloadEncoding

from test_radiance import mixed_bits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("encoding", [PayloadEncoding.RAW, PayloadEncoding.SHUFFLE_LZ4, PayloadEncoding.SHUFFLE_ZSTD])
def test_encode_device_matches_host_encoder(backend, encoding):
    import torch

    fs = workloads.round_brilliant_frame(96, 64)
    sums = np.zeros((64, 96, 3))
    assert backend.try_accumulate(fs, 0, 8, sums)
    for s in (sums, np.random.default_rng(2).random((5, 7, 3)) * 1e3):
        h, w = s.shape[:2]
        d = torch.from_numpy(np.ascontiguousarray(s)).cuda()
        got = rad.encode_device(backend, encoding, d.data_ptr(), w, h)
        want = PayloadEncoder(encoding).encode(s.astype(np.float32).tobytes())
        assert got.encoding == want.encoding and got.raw_len == want.raw_len
        assert got.bytes == want.bytes


@pytest.mark.parametrize("encoding", [PayloadEncoding.RAW, PayloadEncoding.SHUFFLE_LZ4])
def test_decode_and_add_device_matches_host(backend, encoding):
    import torch

    for (w, h), seed in [((1, 1), 3), ((37, 19), 4), ((256, 128), 5)]:
        delta = np.frombuffer(mixed_bits(w * h * 3, seed).tobytes(), np.float32)
        p = PayloadEncoder(encoding).encode(delta.tobytes())
        start = np.random.default_rng(seed).random((h * w, 3), np.float32)
        host = start.copy()
        dropped_h = PayloadDecoder().decode_and_add(p.encoding, p.raw_len, p.bytes, w, h, host)
        d_acc = torch.from_numpy(start.copy()).cuda()
        dropped_d = rad.decode_and_add_device(backend, p.encoding, p.raw_len, p.bytes, w, h, d_acc.data_ptr())
        assert dropped_d == dropped_h
        assert np.array_equal(d_acc.cpu().numpy().view(np.uint32), host.view(np.uint32))


def test_device_decode_checks_like_the_host(backend):
    import torch

    d_acc = torch.zeros((4, 3), dtype=torch.float32, device="cuda")
    with pytest.raises(rad.RadianceError) as e:
        rad.decode_and_add_device(backend, PayloadEncoding.SHUFFLE_LZ4, 48, bytes([0xFF] * 64), 2, 2,
                                  d_acc.data_ptr())
    assert e.value.name == "DecompressFailed"
    with pytest.raises(rad.RadianceError) as e:
        rad.decode_and_add_device(backend, PayloadEncoding.RAW, 60, bytes(48), 2, 2, d_acc.data_ptr())
    assert e.value.name == "RawLenMismatch"
    assert not backend.is_lost()
    assert torch.count_nonzero(d_acc).item() == 0
