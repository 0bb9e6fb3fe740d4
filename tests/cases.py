"""Small T-mixer cases shared by the tests, in the oracle's dict form
(keys of oracle.OrcParams).  Sizes are chosen so the CPU oracle runs each in
well under a second per few dozen steps."""
from __future__ import annotations


def sc_tau(tau: float) -> float:
    """The reference's species relaxation time for Schmidt number 3
    (Tmixer.cpp:86-88)."""
    return (0.5 * (((2.0 * tau - 1.0) / 3.0) + 1.0))


def ref_like(inx: int, iny: int, nz: int, mnx: int, mny: int, **kw) -> dict:
    """The reference's parameters on a smaller grid; ia from the reference's
    formula (Tmixer.cpp:1374)."""
    tau = kw.get("tau", 0.6)
    tc = kw.get("tau_c", sc_tau(tau))
    return dict(inx=inx, iny=iny, nz=nz, mnx=mnx, mny=mny, ia=((inx + 1) // 2) - ((mnx - 1) // 2),
                tau=tau, taua=tc, taub=tc, taup=tc, rho0=kw.get("rho0", 3.0), rho_out=kw.get("rho_out", 3.0),
                c0=0.0, cin=kw.get("cin", [[1.0, 0.0], [0.0, 1.0], [0.0, 0.0]]),
                rateconst=kw.get("k", 1.0), umean=kw.get("umean", 0.059761),
                sc_formula="tau_c" not in kw)


def w_like(W: int, umean: float, tau: float, tau_c: float, k: float, rho: float) -> dict:
    """The benchmark layout of width W (inlet 8W x W x W, mixing 2W x 4W x W)."""
    d = ref_like(8 * W, W, W, 2 * W, 4 * W, tau=tau, tau_c=tau_c, k=k, rho0=rho, rho_out=rho, umean=umean)
    assert d["ia"] == 3 * W + 1
    return d


def ref_params(case: dict) -> dict:
    """Parameters for oracle/build_ref.py (the reference supports one species
    relaxation time and its own ia formula only)."""
    assert case["taua"] == case["taub"] == case["taup"]
    assert case["ia"] == ((case["inx"] + 1) // 2) - ((case["mnx"] - 1) // 2)
    cin = case["cin"]
    return dict(inx=case["inx"], iny=case["iny"], nz=case["nz"], mnx=case["mnx"], mny=case["mny"],
                tau=case["tau"], tau_c=None if case.get("sc_formula") else case["taua"],
                umean=case["umean"], rateconst=case["rateconst"], rho0=case["rho0"], rho_out=case["rho_out"],
                ca_in1=cin[0][0], ca_in2=cin[0][1], cb_in1=cin[1][0], cb_in2=cin[1][1],
                cp_in1=cin[2][0], cp_in2=cin[2][1])


def to_spec(case: dict):
    """The same case as a tmixer_b200.CaseSpec."""
    import tmixer_b200

    return tmixer_b200.CaseSpec(inx=case["inx"], iny=case["iny"], nz=case["nz"], mnx=case["mnx"],
                                mny=case["mny"], ia=case["ia"], tau=case["tau"], tau_a=case["taua"],
                                tau_b=case["taub"], tau_c=case["taup"], rho0=case["rho0"],
                                rho_out=case["rho_out"], c_in=case["cin"], rateconst=case["rateconst"],
                                umean=case["umean"])


# Cases pinned against the reference itself (tests/golden/*.npz).
GOLDEN_CASES = {
    "tiny_ref": (ref_like(21, 7, 7, 7, 14), 40),
    "shrunk_ref": (ref_like(41, 11, 11, 11, 40), 101),
    "w4": (w_like(4, umean=0.03, tau=0.56, tau_c=0.6, k=0.5, rho=1.0), 60),
    "tiny_species": (ref_like(21, 7, 7, 7, 14, tau=0.7, tau_c=0.55, k=3.0, rho0=2.0, rho_out=1.9,
                              cin=[[1.0, 0.25], [0.3, 1.0], [0.1, 0.05]], umean=0.04), 30),
}

# Extra cases only the oracle can run (parameters the reference cannot take).
ORACLE_CASES = {
    "odd_ia": dict(ref_like(24, 6, 5, 8, 9, tau=0.65, k=2.0, rho0=1.5, rho_out=1.4, umean=0.05,
                            cin=[[0.9, 0.2], [0.1, 1.1], [0.05, 0.0]]), ia=6, taua=0.55, taub=0.62, taup=0.7),
    "min3": dict(ref_like(8, 3, 3, 3, 3, tau=0.6, k=1.0, umean=0.02), ia=3),
    # the opening next to both inlet faces (ia = 2, ib = 6); pinned against
    # the reference itself in test_oracle_vs_ref.py
    "wide_opening": ref_like(7, 4, 4, 5, 5, umean=0.03),
}
