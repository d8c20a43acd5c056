"""lbm_pattern_ceiling: every memory pattern runs and reports a positive rate."""
import pytest

import oracle_lib as O

pkg = O.pkg
pytestmark = pytest.mark.gpu

PATTERNS = [(p, pkg.STORE_F32) for p in (pkg.PATTERN_COPY, pkg.PATTERN_PULL, pkg.PATTERN_AA_LOCAL,
                                        pkg.PATTERN_AA_NEIGHBOR, pkg.PATTERN_AA_LOCAL_V8,
                                        pkg.PATTERN_AA_LOCAL_V16)] + \
           [(p, pkg.STORE_F16_SHIFT) for p in range(12)]


@pytest.mark.parametrize("pattern,storage", PATTERNS)
def test_pattern_ceiling_runs(pattern, storage):
    m, g = pkg.pattern_ceiling(pattern, storage, n=64, iters=2)
    assert m > 0 and g > 0
    # bytes per node of the pattern: 2 * 19 * element size
    assert abs(g / m - 2 * 19 * (4 if storage == pkg.STORE_F32 else 2) / 1e3) < 1e-9 * g
