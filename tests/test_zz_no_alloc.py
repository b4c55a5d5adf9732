"""wqc_expectation_pauli_noalloc: Pauli expectations without device allocation.

This entry point serves callers that cannot let a library call cudaMalloc:
hosts whose own allocator already owns the GPU's memory (here, PyTorch's
caching allocator holds the MPS), where cudaMalloc may fail although their
pool has room and cudaFree would synchronise the whole device.  It takes its
working memory from one fixed array inside the library instead.

The GPU test runs the state through the allocating path, copies its sites
into a buffer that torch owns, and checks that the allocation-free entry
point, called three times in a row through the C ABI, gives what
wqc_mps_expectation_pauli gives, within the amplitude tolerance of the
parity tests.  The first call is at bond 256 with six terms, more than the
four that one launch holds at that bond, so the second launch of that call
reuses the environment slots of the first; the later calls use smaller
states and other terms.  Every launch clears the per-term results before it
runs and each transfer-matrix step writes the environment entries it then
reads, so what the calls check is the results clearing, the chunking and the
size bookkeeping, not a full wipe of the array.

The file name sorts last so that a run stopping at its first failure has run
every other test before this one.
"""
import numpy as np
import pytest

import wqc_cuda as W
from wqc_cuda import circuits as C

RTOL = 1e-10  # the parity tests' amplitude tolerance, relative to max(1, |value|)


def random_terms(n: int, count: int, seed: int):
    rng = np.random.Generator(np.random.PCG64(seed))
    labels = ["I" * n] + ["".join(rng.choice(list("IXYZ"), size=n)) for _ in range(count - 1)]
    coeffs = rng.normal(size=count) + 1j * rng.normal(size=count)
    coeffs[0] = 1.0  # the squared norm keeps the sum away from zero
    return labels, coeffs


def caller_owned_sites(m, stride: int):
    """The state's sites copied into a torch buffer at `stride` complex values per site."""
    import torch

    buf = torch.zeros((m.n, stride), dtype=torch.complex128, device="cuda")
    for q in range(m.n):
        s = m.site(q).reshape(-1)
        buf[q, : s.size] = torch.from_numpy(s).to("cuda")
    torch.cuda.synchronize()
    return buf


@pytest.mark.gpu
def test_noalloc_expectation_matches_allocating_entry_point_on_two_calls(cuda_ctx):
    import torch

    stream = torch.cuda.current_stream().cuda_stream
    cases = []
    gates = C.gates_array(C.ry_rz_brickwork(18, 18, seed=10))  # bonds up to 256
    labels, coeffs = random_terms(18, 6, seed=9)  # two launches: 4 terms per launch at bond 256
    cases.append((18, 256, gates, labels, coeffs, 256 * 2 * 256))
    gates = C.gates_array(C.random_layers(14, 10, seed=11))  # bonds up to 64
    labels, coeffs = C.zz_x_observable(14)
    labels, coeffs = labels + ["I" * 14], np.concatenate([coeffs, [1.0]])
    cases.append((14, 64, gates, labels, coeffs, 64 * 2 * 64))
    gates, _, _ = C.hea_ansatz(10, 3, seed=12)  # bonds up to 8
    labels, coeffs = random_terms(10, 70, seed=13)  # more terms than one launch holds
    cases.append((10, 16, gates, labels, coeffs, None))
    bonds = []
    for n, chi, gates, labels, coeffs, stride in cases:
        m = W.CudaMps(n, chi, ctx=cuda_ctx)
        m.apply_gates(gates)
        dims = m.bond_dims()
        bonds.append(int(dims.max()))
        left = np.concatenate([[1], dims[:-1]])
        if stride is None:  # packed as tightly as the largest site allows
            stride = int(np.max(left * 2 * dims))
        buf = caller_owned_sites(m, stride)
        want = m.expectation(labels, coeffs)
        got = W.expectation_pauli_noalloc(buf.data_ptr(), stride, dims, labels, coeffs, stream=stream)
        assert abs(got - want) <= RTOL * max(1.0, abs(want)), (n, chi, got, want)
        assert abs(want) > 1e-3  # the comparison is not between two zeros
    assert bonds[0] == 256 and bonds[0] > bonds[1] > bonds[2]  # each call reads less than the one before wrote


def test_noalloc_expectation_rejects_sizes_beyond_its_limits():
    # Sizes are checked before any device work, so this runs without a GPU.
    with pytest.raises(W.WqcCudaError) as e:
        W.expectation_pauli_noalloc(0, 2 * 257 * 2, [2, 257, 1], ["ZZZ"], [1.0])
    assert e.value.code == W.ERR_INVALID and "256" in str(e.value)
    with pytest.raises(W.WqcCudaError) as e:
        W.expectation_pauli_noalloc(0, 2, [1] * 1025, ["Z" * 1025], [1.0])
    assert e.value.code == W.ERR_INVALID_QUBIT_COUNT and "1024" in str(e.value)
    with pytest.raises(W.WqcCudaError) as e:
        W.expectation_pauli_noalloc(0, 4, [2, 2, 1], ["ZZZ"], [1.0])  # site 1 is 2x2x2 = 8 > 4
    assert e.value.code == W.ERR_INVALID and "stride" in str(e.value)


def test_noalloc_expectation_rejects_an_open_chain():
    # The recursion's result is the expectation only when the last right bond
    # is 1; a trailing bond above 1 is refused before any device work.
    with pytest.raises(W.WqcCudaError) as e:
        W.expectation_pauli_noalloc(0, 8, [2, 2, 2], ["ZZZ"], [1.0])
    assert e.value.code == W.ERR_INVALID and "closed chain" in str(e.value)
