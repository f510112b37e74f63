"""Host-side parts of xnyzip_b200.verify (the checks bench.py and the GPU tests apply to
decoded clouds): the multiset comparison through point hashes, the float32 slack, SHA-256 of
tensors and arrays."""
import hashlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def test_multiset_mismatch_counts_unmatched_points():
    from xnyzip_b200.verify import multiset_mismatch
    g = torch.Generator().manual_seed(3)
    a = torch.randn((5000, 3), generator=g)
    a[100:200] = a[0]  # repeated points count with multiplicity
    b = a[torch.randperm(5000, generator=g)].clone()
    assert multiset_mismatch(a, b) == 0
    b[7, 2] = 1e6
    b[9] = b[11]
    assert multiset_mismatch(a, b) == 2
    c = a[torch.randperm(5000, generator=g)][:4000]
    assert multiset_mismatch(a, c) == 1000


def test_f32_slack_follows_float_resolution():
    from xnyzip_b200.verify import f32_slack
    small = torch.tensor([[0.0, 0.0, 0.0], [10.0, 10.0, 1.0]])
    big = torch.tensor([[0.0, 0.0, 0.0], [10000.0, 10000.0, 100.0]])
    assert f32_slack(small, 1, 0.01) < 1e-5
    # 10 km at a 1 mm bound: the lattice index alone is rounded to whole steps
    assert 0.003 < f32_slack(big, 1, 0.001) < 0.01
    assert f32_slack(big[:0], 0, 0.1) == 0.0


def test_sha256_of_tensors_and_arrays():
    from xnyzip_b200.verify import sha256
    x = np.arange(30, dtype=np.float32).reshape(10, 3)
    want = hashlib.sha256(x.tobytes()).hexdigest()
    assert sha256(x) == want == sha256(torch.from_numpy(x)) == sha256(x.tobytes())
