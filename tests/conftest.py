import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the CUDA kernels")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def qb():
    import quoin_b200 as Q
    return Q


M64 = (1 << 64) - 1


def lcg_seq(seed: int, n: int):
    """The reference tests' LCG (tests/roundtrip.rs:58-63): s = s*6364136223846793005 + 1442695040888963407."""
    import numpy as np
    out = np.empty(n, dtype=np.uint64)
    s = seed
    for i in range(n):
        s = (s * 6364136223846793005 + 1442695040888963407) & M64
        out[i] = s
    return out


def lcg1_seq(seed: int, n: int):
    """The reference unit tests' LCG with increment 1 (e.g. bitpack.rs:206-212 uses
    6364136223846793005 / 1442695040888963407; dict.rs / for_bitpack.rs use +1)."""
    import numpy as np
    out = np.empty(n, dtype=np.uint64)
    s = seed
    for i in range(n):
        s = (s * 6364136223846793005 + 1) & M64
        out[i] = s
    return out


def bitmap_from_bools(bits):
    import numpy as np
    bits = np.asarray(bits, dtype=bool)
    n = bits.size
    return np.packbits(bits, bitorder="little") if n else np.zeros(0, dtype=np.uint8)
