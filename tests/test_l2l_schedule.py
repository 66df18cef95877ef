"""The mixed L2L's balanced product list (k_l2l_mixed in fmms_b200/csrc/mixed.cu).

The kernel lays the products of all outputs of one L2L out as one list and
gives every lane of a warp an equal run of it; outputs that cross runs are
summed from per-lane partial slots afterwards. This restates the list and the
run/slot rules in Python and checks, for every order the mixed form runs
(p <= 16), that the packed fields fit their bits and that every output gets
exactly its own products, each once, with no partial slot written twice.
"""

import pytest

LAST = 1 << 31


def l2l_items(p):
    return (p + 1) * (p + 2) * (p + 2) * (p + 3) // 12


def build(p):
    """(items, einfo) as the kernel's blocks build them."""
    H = (p + 1) * (p + 2) // 2
    T = l2l_items(p)
    items = [None] * T
    einfo = [0] * (H + 1)
    for e in range(H):
        n = 0
        while (n + 1) * (n + 2) // 2 <= e:
            n += 1
        m = e - n * (n + 1) // 2
        s = sum((q + 1) * (p - q + 1) ** 2 for q in range(n)) + m * (p - n + 1) ** 2
        einfo[e] = s | (n << 16)
        for k in range(p - n + 1):
            for l in range(-k, k + 1):
                ui = k * (k + 1) + l
                fi = (n + k) * (n + k + 1) + m + l
                assert 0 <= ui < 512 and 0 <= fi < 512 and e < 256
                assert items[s] is None
                items[s] = ui | (fi << 9) | (e << 18) | (LAST if (k == p - n and l == k) else 0)
                s += 1
    einfo[H] = T
    assert all(it is not None for it in items)
    assert T < 1 << 16
    return items, einfo


def run_warp(items, einfo, vals):
    """Per-output sums through the lanes' runs, partial slots and lane-order combine."""
    T = len(items)
    H = len(einfo) - 1
    W = ((T + 31) // 32) | 1
    R = [None] * H
    slots = [[None, None] for _ in range(32)]

    def put(lane, slot, v):
        assert slots[lane][slot] is None
        slots[lane][slot] = v

    for lane in range(32):
        r0 = min(T, lane * W)
        r1 = min(T, r0 + W)
        acc, it = [], None
        for i in range(r0, r1):
            it = items[i]
            acc.append(vals[i])
            if it & LAST:
                e = (it >> 18) & 255
                if (einfo[e] & 0xFFFF) >= r0:
                    assert R[e] is None
                    R[e] = acc
                else:
                    put(lane, 0, acc)
                acc = []
        if r1 > r0 and not (it & LAST):
            e = (it >> 18) & 255
            put(lane, 0 if (einfo[e] & 0xFFFF) <= r0 else 1, acc)
    for lane in range(32):
        r0 = min(T, lane * W)
        r1 = min(T, r0 + W)
        if r1 > r0:
            e = (items[r1 - 1] >> 18) & 255
            s0, s1 = einfo[e] & 0xFFFF, einfo[e + 1] & 0xFFFF
            if s0 >= r0 and s1 > r1:
                acc = list(slots[lane][0 if s0 == r0 else 1])
                q = lane + 1
                while q * W < s1:
                    acc += slots[q][0]
                    q += 1
                assert R[e] is None
                R[e] = acc
    return R


@pytest.mark.parametrize("p", list(range(0, 17)))
def test_every_output_gets_exactly_its_products(p):
    items, einfo = build(p)
    T = len(items)
    H = len(einfo) - 1
    assert T == sum((n + 1) * (p - n + 1) ** 2 for n in range(p + 1))
    R = run_warp(items, einfo, list(range(T)))  # product i contributes its own index
    for e in range(H):
        lo, hi = einfo[e] & 0xFFFF, einfo[e + 1] & 0xFFFF
        assert R[e] is not None
        assert sorted(R[e]) == list(range(lo, hi)), (p, e)
        # lane order: the products arrive in list order, so the sum order is fixed
        assert R[e] == list(range(lo, hi)), (p, e)
