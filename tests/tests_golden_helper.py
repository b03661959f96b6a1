"""Helper shared by tests: where the reference's own level count is defined."""
import math


def ref_level_count_ok(n: int, b: int) -> bool:
    hf = int(math.log10(n) / math.log10(b + 1))
    h, p = 0, 1
    while p * (b + 1) <= n:
        p *= b + 1
        h += 1
    return hf == h
