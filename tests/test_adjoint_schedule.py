"""The bounded-memory schedule of the transient CUDA adjoint (tnsgpu.adjoint._Checkpoints)
on a stand-in device: every reverse step sees the state of its own iteration, in the
order N-1 .. 0, and no more than ``max_states`` states are held at once."""
import pytest

from tnsgpu.adjoint import _Checkpoints


class _Pool:
    def __getitem__(self, k):
        return k


class _Dev:
    def __init__(self):
        self.solver = None

    def _enter(self):
        pass

    def _leave(self):
        pass


def _run(N, cap):
    dev = _Dev()
    cp = _Checkpoints.__new__(_Checkpoints)
    cp.dev, cp.cap, cp.recomputed = dev, cap, 0
    cp.free = list(range(cap - 1, -1, -1))
    cp.pool = _Pool()
    held = {}
    peak = [0]

    def advance(src, n, dst):
        held[dst] = held[src] + n
        cp.recomputed += n
        peak[0] = max(peak[0], cap - len(cp.free))

    cp.advance = advance
    seen = []
    dev.step = lambda slot, lam, sens: seen.append(held[slot])
    root = cp.take()
    held[root] = 0
    cp.sweep(0, N, root, None, True)
    return seen, cp.recomputed, peak[0]


@pytest.mark.parametrize("N,cap", [(1, 2), (7, 2), (30, 2), (30, 4), (30, 31), (500, 16), (1000, 5)])
def test_every_iteration_is_reversed_in_order_within_the_slot_budget(N, cap):
    seen, recomputed, peak = _run(N, cap)
    assert seen == list(range(N - 1, -1, -1))
    assert peak <= cap
    assert recomputed >= N - 1


def test_recomputation_grows_like_n_log_n():
    # the c4 transient: 10 000 iterations with 64 state slots
    _, recomputed, peak = _run(10000, 64)
    assert recomputed < 6 * 10000 and peak <= 64
