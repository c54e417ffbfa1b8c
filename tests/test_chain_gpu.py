"""Device-resident chains on the GPU: M = X_0 X_1 ... with the running
product kept in device memory between steps.  Results are compared
bit-exactly with the golden digest of the config-2 chain (16 signed 8x8
matrices of 65536-bit entries, computed by the reference and GMP), with the
same chain through host round trips, and with Python integers."""
import random

import pytest

from rforest_b200 import _lib, api, packed as PK, workloads as W
from tests import golden_io as G

pytestmark = pytest.mark.gpu


def python_chain(mats):
    rows, _, X = mats[0]
    M = [X.entry(e) for e in range(len(X))]
    cols = mats[0][1]
    for r, c, Y in mats[1:]:
        Yi = [Y.entry(e) for e in range(len(Y))]
        M = [sum(M[i * cols + l] * Yi[l * c + j] for l in range(cols))
             for i in range(rows) for j in range(c)]
        cols = c
    return M


def test_config2_chain_golden(gpu):
    d = G.digests()["config2_chain"]
    mats = W.config2_chain()
    C = api.chain([(8, 8, X) for X in mats])
    assert PK.digest(C) == d["steps"][-1]
    # the first steps as shorter chains
    for steps in (1, 2, 5):
        C = api.chain([(8, 8, X) for X in mats[:steps + 1]])
        assert PK.digest(C) == d["steps"][steps - 1], f"{steps} steps"


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_chains_vs_python(gpu, seed):
    rng = random.Random(seed)
    for _ in range(6):
        dims = [rng.randrange(1, 6) for _ in range(rng.randrange(3, 6))]
        mats = []
        for i in range(len(dims) - 1):
            bits = rng.choice([1, 60, 64, 65, 300, 2000, 9000])
            vals = [rng.choice([0, 1, -1, 1, -1]) * rng.getrandbits(bits)
                    for _ in range(dims[i] * dims[i + 1])]
            if not any(vals):
                vals[0] = 1
            mats.append((dims[i], dims[i + 1], PK.from_ints(vals)))
        C = api.chain(mats)
        assert C.to_ints() == python_chain(mats), dims


def test_chain_equals_host_round_trips(gpu):
    rng = random.Random(11)
    mats = []
    for i in range(6):
        vals = [rng.choice([1, -1]) * rng.getrandbits(rng.choice([500, 4000, 20000]))
                for _ in range(16)]
        mats.append((4, 4, PK.from_ints(vals)))
    M = mats[0][2]
    for _, _, X in mats[1:]:
        M = api.matmul(4, 4, 4, M, X).compact()
    assert PK.digest(api.chain(mats)) == PK.digest(M)


def test_chain_zero_factor_and_errors(gpu):
    A = PK.from_ints([3, -4, 5, 6])
    Z = PK.from_ints([0, 0, 0, 0])
    C = api.chain([(2, 2, A), (2, 2, Z), (2, 2, A)])
    assert C.to_ints() == [0, 0, 0, 0]
    with pytest.raises(_lib.MpzmmError) as e:
        api.chain([(2, 2, A), (3, 1, PK.from_ints([1, 2, 3]))])
    assert e.value.status == _lib.MPZMM_ERR_ARG
    with pytest.raises(_lib.MpzmmError):
        api.chain([(2, 2, A)])
