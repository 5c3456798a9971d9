"""The autotuner's search space (tune.py) without a GPU: which tiles and schedules are timed for
each sequence, and the cache key."""
from cuda_ultrasound_toolkit_b200 import SequenceId, synth
from cuda_ultrasound_toolkit_b200 import tune


def bp_of(seq, same_orientation=False):
    bp = synth.make_params(synth.CONFIGS["small"])
    bp.das_shader_id = int(seq)
    if same_orientation:
        bp.tx_orientation = bp.rx_orientation
    return bp


def test_search_space_per_sequence():
    herc = bp_of(SequenceId.HERCULES)
    assert tune.candidates(herc) == (1, 2)
    assert all(tune.schedules(herc, t) == (0, 2) for t in (1, 2))
    tpw_yz = bp_of(SequenceId.RCA_TPW)
    assert tune.candidates(tpw_yz) == (1, 2, 3)
    assert tune.schedules(tpw_yz, 2) == (0, 1, 2) and tune.schedules(tpw_yz, 3) == (0,)
    assert tune.candidates(bp_of(SequenceId.RCA_TPW, True)) == (2, 3)
    assert tune.candidates(bp_of(SequenceId.UFORCES, True)) == (2, 3)
    forces = bp_of(SequenceId.FORCES, True)
    assert tune.candidates(forces) == (0,) and tune.schedules(forces, 0) == (0, 1, 2)
    assert tune.ROWS[0] == 8 and all(1 <= r <= 8 for r in tune.ROWS)


def test_key_separates_what_changes_the_work():
    a, b = bp_of(SequenceId.HERCULES), bp_of(SequenceId.HERCULES)
    assert tune.key(a) == tune.key(b)
    b.coherency_weighting = 1.0
    assert tune.key(a) != tune.key(b)
    assert tune.key(a) != tune.key(a, iq_bf16=True)
    assert tune.config_name(2, 0, 4) == "tile2/schedule0/rows4"
