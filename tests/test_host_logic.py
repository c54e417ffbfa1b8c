"""Host-side helpers on the CPU: exact bit lengths of packed operands (they
size the output arrays the library writes straight into)."""
import random

import numpy as np

from rforest_b200 import packed as PK


def test_bit_length_u64_exact():
    rng = random.Random(1)
    vals = [0, 1, 2, 3, 1 << 63, (1 << 64) - 1, (1 << 53) - 1, 1 << 53, (1 << 53) + 1]
    vals += [rng.getrandbits(rng.randrange(1, 65)) for _ in range(2000)]
    got = PK.bit_length_u64(np.array(vals, dtype=np.uint64))
    assert [int(b) for b in got] == [v.bit_length() for v in vals]


def test_packed_max_bits():
    rng = random.Random(2)
    for _ in range(50):
        vals = [rng.choice([0, 1, -1]) * rng.getrandbits(rng.randrange(0, 700))
                for _ in range(rng.randrange(0, 12))]
        P = PK.from_ints(vals)
        assert P.max_bits() == max((abs(v).bit_length() for v in vals), default=0)
