"""The default gravity walk by problem size (gpop_walk_policy, the function the propagation
launches follow), checked at the boundaries of its bands on a 148-SM B200: lanes up to 128
objects per SM (lanes per object chosen so a block has at most 384 threads), FP64 two lanes per
object up to 192 per SM, then FP64 one object per thread up to 256 per SM, and two objects per
thread above (mixed precision from 128 per SM). Host arithmetic only: runs without a GPU."""
import pytest

SMS = 148


def test_walk_bands():
    import opengpop_b200 as G
    W = G.walk_policy
    per = lambda k: k * SMS  # objects at k per SM
    for prec in (G.FP64, G.MIXED):
        assert W(1, SMS, prec) == (3, 32)
        assert W(per(128), SMS, prec)[0] == 3
    assert W(per(128) + 1, SMS, G.MIXED) == (2, 1)
    assert W(per(128) + 1, SMS, G.FP64) == (3, 2)
    assert W(per(192), SMS, G.FP64) == (3, 2)
    assert W(per(192) + 1, SMS, G.FP64) == (1, 1)
    assert W(per(256), SMS, G.FP64) == (1, 1)
    assert W(per(256) + 1, SMS, G.FP64) == (2, 1)
    assert W(65536, SMS, G.MIXED) == (2, 1) and W(65536, SMS, G.FP64) == (2, 1)


def test_lane_blocks_fit_the_register_variant():
    # wherever the default walk takes lanes, one block of at most 384 threads per SM holds them
    import opengpop_b200 as G
    for prec in (G.FP64, G.MIXED):
        for n in list(range(1, 4096, 7)) + list(range(4096, 30000, 97)):
            w, P = G.walk_policy(n, SMS, prec)
            if w == 3:
                per_sm = -(-n * P // SMS)
                assert -(-per_sm // 32) * 32 <= 384, (n, prec, P)
                assert P == 32 or 2 * P * n > SMS * 384, (n, P)  # the most lanes that fit


def test_walk_policy_rejects_bad_arguments():
    import opengpop_b200 as G
    for args in ((0, SMS, G.FP64), (10, 0, G.FP64), (10, SMS, 7)):
        with pytest.raises(G.GpopError):
            G.walk_policy(*args)
