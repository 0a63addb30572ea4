"""The objective bar of the parity tests, shared by every file that compares a solve with the
reference's (or with another solve of the same problem)."""


def objectives_close(pobj, dobj, ref_pobj, ref_dobj, tol=1e-7, each=False):
    """Objectives within `tol` relative:
    - the optimal-value estimate (pobj + dobj) / 2 plainly relative, |v - v_ref| <= tol max(1, |v_ref|)
      (the floor of 1 keeps the bar finite for objectives at 0), always;
    - pobj and dobj each plainly relative in the same way, when `each`: the callers set it when
      the solve ended at the reference's own iteration count (the same iterate up to rounding);
    - pobj and dobj each within tol of the DIMACS gap's denominator 1 + |pobj_ref| + |dobj_ref|,
      always.  This is the accuracy either solve has at DIMACS error tol: two solves that both
      meet the tolerance bracket the optimum with gaps of up to tol times that denominator, so
      their pobj (or dobj) may differ by that much while their (pobj + dobj) / 2 agree.  That is
      the case when one solve stops an iteration before the other (rand60: the reference's 12th
      iteration took its gap from 6e-8 to 5e-9, this build stopped at 11 with 6.5e-8), or when it
      computes in another order (the lockstep batch).
    Raises AssertionError naming the value that misses."""
    den = 1 + abs(ref_pobj) + abs(ref_dobj)
    mid, ref_mid = 0.5 * (pobj + dobj), 0.5 * (ref_pobj + ref_dobj)
    assert abs(mid - ref_mid) <= tol * max(1.0, abs(ref_mid)), ("(pobj + dobj) / 2", mid, ref_mid)
    for name, got, want in (("pobj", pobj, ref_pobj), ("dobj", dobj, ref_dobj)):
        if each:
            assert abs(got - want) <= tol * max(1.0, abs(want)), (name, got, want)
        assert abs(got - want) <= tol * den, (name, got, want)
