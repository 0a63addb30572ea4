"""The objective bar of the parity tests, shared by every file that compares a solve with the
reference's (or with another solve of the same problem)."""


def objectives_close(pobj, dobj, ref_pobj, ref_dobj, tol=1e-7):
    """Objectives within `tol` relative, checked two ways:
    - as the north star states it, plainly relative: |obj - obj_ref| <= tol max(1, |obj_ref|)
      (the floor of 1 keeps the bar finite for objectives at 0);
    - relative to the DIMACS gap's denominator 1 + |pobj_ref| + |dobj_ref|: the accuracy either
      solve has at DIMACS error tol, looser than the first when |pobj| ~ |dobj| >> 1, kept as the
      stated reason why two solves that both meet the tolerance may differ by that much.
    Raises AssertionError naming the pair that misses."""
    den = 1 + abs(ref_pobj) + abs(ref_dobj)
    for name, got, want in (("pobj", pobj, ref_pobj), ("dobj", dobj, ref_dobj)):
        assert abs(got - want) <= tol * max(1.0, abs(want)), (name, got, want)
        assert abs(got - want) <= tol * den, (name, got, want)
