"""Feet and actions of the labelling fixture (tests/golden/labels.npz): (name, Foot fields, Action fields,
defect_fill), chosen to reach every branch of rb/rbgeom.py:358-464."""

LABEL_CASES = [
    ("default", {}, {}, "soft"),
    ("scaled", dict(scale=1.08), {}, "soft"),
    ("facets_ant1", dict(post_a=14.0, post_b=8.0, mid_a=5.0, mid_b=5.5, ant_a=5.5, ant_mode=1), {}, "soft"),
    ("ant2", dict(ant_mode=2, mid_a=7.5), {}, "soft"),
    ("warps", dict(sust_y=14.0, post_dome=3.0), {}, "soft"),
    ("valgus", dict(align=8.0, scale=0.95), {}, "soft"),
    ("R1", dict(ctype="I", rtype="R1", cov_mid=0.4), {}, "soft"),
    ("R2", dict(ctype="I", rtype="R2", cov_mid=0.3), {}, "soft"),
    ("R3", dict(ctype="I", rtype="R3", cov_mid=0.5, fib_frac=0.5), {}, "soft"),
    ("R4", dict(ctype="I", rtype="R4", cov_mid=0.6, seed_ang=20.0), {}, "soft"),
    ("II", dict(ctype="II", cov_post=0.35), {}, "void"),
    ("III", dict(ctype="III"), {}, "soft"),
    ("IV_resect", dict(ctype="IV", rtype="R1", cov_mid=0.5, cov_post=0.2), dict(resect=1, d_mid=0.3, d_post=0.2), "soft"),
    ("IV_interp", dict(ctype="IV", cov_mid=0.4, cov_post=0.3), dict(resect=1, interp=1, d_mid=0.2), "soft"),
    ("resect_void", dict(ctype="I", rtype="R2", cov_mid=0.4), dict(resect=1, d_post=0.25), "void"),
    ("osteo", dict(post_dome=2.5), dict(osteo=6.0), "soft"),
    ("osteo_lat", dict(align=-5.0), dict(osteo=-4.0), "soft"),
    ("fusion", dict(ctype="II", cov_post=0.5, sust_y=9.0), dict(fusion=1), "soft"),
]
