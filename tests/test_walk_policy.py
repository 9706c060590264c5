"""The default gravity walk by problem size (gpop_walk_policy, the function the propagation
launches follow), checked at the boundaries of its bands on a 148-SM B200: lanes up to 128
objects per SM (lanes per object chosen so a block has at most 384 threads), lanes per group of
two objects where they gain (FP64 from 8 to 150 objects per SM, mixed precision from 16 to 150),
FP64 two lanes per object up to 192 per SM, then FP64 one object per thread up to 256 per SM, and
two objects per thread above (mixed precision from 150 per SM). Host arithmetic only: runs
without a GPU."""
import pytest

SMS = 148


def test_walk_bands():
    import opengpop_b200 as G
    W = G.walk_policy
    per = lambda k: k * SMS  # objects at k per SM
    for prec in (G.FP64, G.MIXED):
        assert W(1, SMS, prec) == (3, 32)
        assert W(per(128), SMS, prec) == (4, 4)
        assert W(per(150), SMS, prec) == (4, 4)
    assert W(per(150) + 1, SMS, G.MIXED) == (2, 1)
    assert W(per(150) + 1, SMS, G.FP64) == (3, 2)
    assert W(per(192), SMS, G.FP64) == (3, 2)
    assert W(per(192) + 1, SMS, G.FP64) == (1, 1)
    assert W(per(256), SMS, G.FP64) == (1, 1)
    assert W(per(256) + 1, SMS, G.FP64) == (2, 1)
    assert W(65536, SMS, G.MIXED) == (2, 1) and W(65536, SMS, G.FP64) == (2, 1)


def test_lane_pair_bands():
    # two objects per lane group: the most lanes whose groups fit one wave of 8 warps per SM,
    # doubled once up to 8 lanes when the groups still fit 1.5 waves (FP64) or 1.2 waves (mixed)
    import opengpop_b200 as G
    W = G.walk_policy
    per = lambda k: k * SMS
    assert W(per(8) - 1, SMS, G.FP64)[0] == 3 and W(per(8), SMS, G.FP64) == (4, 32)
    assert W(4096, SMS, G.FP64) == (4, 16) and W(6000, SMS, G.FP64) == (4, 8)
    assert W(9472, SMS, G.FP64) == (4, 8) and W(12000, SMS, G.FP64) == (4, 8)
    assert W(14000, SMS, G.FP64) == (4, 8) and W(16000, SMS, G.FP64) == (4, 4)
    assert W(20000, SMS, G.FP64) == (4, 4) and W(22000, SMS, G.FP64) == (4, 4)
    assert W(per(16) - 1, SMS, G.MIXED)[0] == 3 and W(per(16), SMS, G.MIXED) == (4, 32)
    assert W(6000, SMS, G.MIXED) == (4, 8) and W(12000, SMS, G.MIXED) == (4, 4)
    assert W(9472, SMS, G.MIXED) == (4, 8) and W(20000, SMS, G.MIXED) == (4, 4)
    for prec in (G.FP64, G.MIXED):
        for n in range(1, per(200), 37):
            w, P = W(n, SMS, prec)
            if w == 4:  # the first launch holds at most one wave of 8 warps per SM
                main = min(n, SMS * 256 // P * 2)
                assert -(-main // 2) * P <= SMS * 256, (n, P)


def test_split_block_bands():
    # two objects per thread with 5 to 7 sets of 64 objects per SM take the split block (owner
    # warps = sets); 8 sets fill the plain block, and degree 8 or less has no FP32 tail to split
    import opengpop_b200 as G
    per = lambda k: k * SMS
    assert G.split_block(per(256), SMS) == 0
    assert G.split_block(per(256) + 1, SMS) == 5
    assert G.split_block(per(320), SMS) == 5 and G.split_block(per(320) + 1, SMS) == 6
    assert G.split_block(per(384), SMS) == 6 and G.split_block(per(384) + 1, SMS) == 7
    assert G.split_block(65536, SMS) == 7 and G.split_block(per(448), SMS) == 7
    assert G.split_block(per(448) + 1, SMS) == 0
    assert G.split_block(65536, SMS, degree=8) == 0 and G.split_block(65536, SMS, degree=9) == 7
    for args in ((0, SMS, 70), (10, 0, 70), (10, SMS, -1)):
        with pytest.raises(G.GpopError):
            G.split_block(*args)


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


@pytest.mark.parametrize("sms", [1, 7, 132, 148, 160])
def test_policy_invariants_for_any_sm_count(sms):
    # whatever the GPU: a split block holds every object of its launch in its owner warps, lane
    # groups have a power-of-two lane count, and the first lane-pair launch fits one wave
    import opengpop_b200 as G
    for prec in (G.FP64, G.MIXED):
        for n in list(range(1, 4000, 13)) + list(range(4000, sms * 700, max(1, sms * 3))):
            w, P = G.walk_policy(n, sms, prec)
            assert w in (1, 2, 3, 4) and P >= 1 and P & (P - 1) == 0 and P <= 32
            S = G.split_block(n, sms)
            assert S == 0 or 5 <= S <= 7
            if S:
                assert 2 * sms * 32 * S >= n
            if w == 4:
                main = min(n, sms * 256 // P * 2)
                assert -(-main // 2) * P <= sms * 256
