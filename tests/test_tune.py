"""Tuner host logic (no GPU): the probe grids it measures each size class on."""


def test_tuner_probe_grids_fall_in_their_size_class():
    """The tuner measures each size class on grids whose cell count lies in
    [2^cls, 2^(cls+1))."""
    from adaptflood_b200.batch import size_class
    from adaptflood_b200.tune import _probe_case
    for cls in range(6, 25):
        c = _probe_case(cls)
        assert 2 ** cls <= c.nx * c.ny < 2 ** (cls + 1)
        assert size_class(c.nx, c.ny) == cls
