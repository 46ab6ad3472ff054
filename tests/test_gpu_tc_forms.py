"""The tensor-core operand forms of hp_tc.cuh, one tcgen05.mma at a time
(hp_tc_check_mma): D [128, 256] = A [128 x 16] * B [256 x 16]^T from operand
images laid out here with the same byte offsets the kernels use, against the
host product.  Entries are small integers, so every product and sum is exact
in bf16 x bf16 -> fp32 and the comparison is equality.

The forms: A 128-byte swizzled (the Aggregator's activations: K blocks of 64,
the descriptor advanced by 32 bytes per 16 K) or no swizzle (its 16-wide
extra-input operand E); B 64-byte swizzled (the streamed weight chunks of
256 x 32 K), no swizzle (block3.0's extra-input weights W3b) or 128-byte
swizzled (the colour branch's chunks).
"""
import zlib

import numpy as np
import pytest
import torch

from hashpoint import native

pytestmark = pytest.mark.gpu

PLAIN, SW128, SW64 = 0, 1, 2


@pytest.fixture(scope="module", autouse=True)
def _setup():
    native.build_testing()


def plain_offset(r, k):
    """Element (r, k), k < 16, of a no-swizzle operand (K-adjacent core matrices 128 bytes apart, row groups 256)."""
    return (r >> 3) * 256 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2


def sw128_offset(r, k, rows):
    """Element (r, k) of a 128-byte-swizzled operand of `rows` rows in K blocks of 64."""
    return (k >> 6) * rows * 128 + r * 128 + ((((k >> 3) & 7) ^ (r & 7)) << 4) + (k & 7) * 2


def sw64_offset(n, k):
    """Element (n, k), k < 32, of a 64-byte-swizzled chunk."""
    return n * 64 + ((((k >> 3) & 3) ^ ((n >> 1) & 3)) << 4) + (k & 7) * 2


def image(mat, form, nbytes):
    """bf16 image (uint8 [nbytes]) of the [rows, K] matrix in the given form."""
    rows, K = mat.shape
    r, k = np.meshgrid(np.arange(rows), np.arange(K), indexing="ij")
    if form == PLAIN:
        off = plain_offset(r, k)
    elif form == SW128:
        off = sw128_offset(r, k, rows)
    else:
        off = sw64_offset(r, k)
    bits = torch.from_numpy(mat.astype(np.float32)).bfloat16().view(torch.int16).numpy().view(np.uint16)
    img = np.zeros(nbytes // 2, np.uint16)
    img[(off // 2).reshape(-1)] = bits.reshape(-1)
    return img.view(np.uint8)


def window_start(form, k0, rows):
    """Descriptor start (bytes) of the 16-wide K window at column k0."""
    if form == PLAIN:
        assert k0 == 0
        return 0
    if form == SW128:
        return (k0 >> 6) * rows * 128 + (k0 & 63) * 2
    assert k0 in (0, 16)
    return k0 * 2


def run_case(a_form, a_k, a_k0, b_form, b_k, b_k0, live, seed):
    """One MMA over A's K columns a_k0.. and B's b_k0..; only the first `live` of the 16 are nonzero."""
    L = native.testing_lib()
    rng = np.random.default_rng(seed)
    A = rng.integers(-3, 4, (128, a_k)).astype(np.float32)
    B = rng.integers(-3, 4, (256, b_k)).astype(np.float32)
    A[:, a_k0 + live:a_k0 + 16] = 0
    B[:, b_k0 + live:b_k0 + 16] = 0
    a_img = torch.from_numpy(image(A, a_form, L.hp_tc_check_image_bytes(0))).cuda()
    b_img = torch.from_numpy(image(B, b_form, L.hp_tc_check_image_bytes(1))).cuda()
    d = torch.empty(128, 256, dtype=torch.float32, device="cuda")
    rc = L.hp_tc_check_mma(a_img.data_ptr(), b_img.data_ptr(), a_form, window_start(a_form, a_k0, 128), b_form,
                           window_start(b_form, b_k0, 256), d.data_ptr(), torch.cuda.current_stream().cuda_stream)
    native.check(rc, "hp_tc_check_mma", L)
    want = A[:, a_k0:a_k0 + 16] @ B[:, b_k0:b_k0 + 16].T
    return d.cpu().numpy(), want


# (name, A form, A width, A window, B form, B width, B window, live K columns): forms the kernels use
USED = [
    ("weights, first K step", SW128, 320, 0, SW64, 32, 0, 16),
    ("weights, K step 16", SW128, 320, 16, SW64, 32, 16, 16),
    ("weights, K step 48", SW128, 320, 48, SW64, 32, 16, 16),
    ("weights, block 4", SW128, 320, 272, SW64, 32, 16, 16),
    ("colour chunk", SW128, 320, 96, SW128, 64, 32, 16),
    ("extras, K 0..7", PLAIN, 16, 0, PLAIN, 16, 0, 8),
]
# forms no kernel relies on yet: A0's padding columns, the no-swizzle operands' upper K half, a swizzled A
# with a no-swizzle B (the operands of a bias folded into the MMAs)
UNUSED = [
    ("A0 padding, K 288", SW128, 320, 288, SW64, 32, 0, 16),
    ("A0 padding, K 304", SW128, 320, 304, SW64, 32, 16, 16),
    ("extras, K 0..15", PLAIN, 16, 0, PLAIN, 16, 0, 16),
    ("swizzled A x plain B", SW128, 320, 288, PLAIN, 16, 0, 16),
]


@pytest.mark.parametrize("case", USED + UNUSED, ids=[c[0] for c in USED + UNUSED])
def test_operand_forms(case):
    name, *spec = case
    got, want = run_case(*spec, seed=zlib.crc32(name.encode()))
    np.testing.assert_array_equal(got, want)


def test_rejects_windows_outside_the_image():
    L = native.testing_lib()
    a = torch.zeros(L.hp_tc_check_image_bytes(0), dtype=torch.uint8, device="cuda")
    b = torch.zeros(L.hp_tc_check_image_bytes(1), dtype=torch.uint8, device="cuda")
    d = torch.empty(128, 256, dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    for a_form, a_off, b_form, b_off in ((SW128, 81920 - 16384 + 112, SW64, 0), (SW128, 8, SW64, 0),
                                         (PLAIN, 81920 - 4096 + 16, SW64, 0), (SW128, 0, SW128, 128), (7, 0, SW64, 0)):
        assert L.hp_tc_check_mma(a.data_ptr(), b.data_ptr(), a_form, a_off, b_form, b_off, d.data_ptr(), s) == -1
