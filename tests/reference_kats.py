"""Known-answer values held by signedMCRT's own test suite (Fortran, test-drive),
transcribed with the file:line of each check.  Paths are relative to the
signedMCRT project root.
"""
import math

R3 = 1.0 / math.sqrt(3.0)
R2 = 1.0 / math.sqrt(2.0)

# (constructor, args, [(point, expected, threshold)])  -- test/SDF/test_SDF.f90
SDF_KATS = [
    ("sphere", dict(radius=1.0), [  # :676-719
        ((0, 0, 0), -1.0, None), ((0, 1, 0), 0.0, None), ((0, 0, 1), 0.0, None), ((1, 0, 0), 0.0, None),
        ((0, -1, 0), 0.0, None), ((0, 0, -1), 0.0, None), ((-1, 0, 0), 0.0, None), ((R3, R3, R3), 0.0, 1e-15)]),
    ("box", dict(lengths=(2.0, 2.0, 2.0)), [  # :721-764
        ((0, 0, 0), -1.0, None), ((0, 1, 0), 0.0, None), ((0, 0, 1), 0.0, None), ((1, 0, 0), 0.0, None),
        ((0, -1, 0), 0.0, None), ((0, 0, -1), 0.0, None), ((-1, 0, 0), 0.0, None), ((1, 1, 1), 0.0, None)]),
    ("cylinder", dict(a=(0, 0, -1), b=(0, 0, 1), radius=1.0), [  # :766-811
        ((0, 0, 0), -1.0, None), ((0, 1, 0), 0.0, None), ((0, 0, 1), 0.0, None), ((1, 0, 0), 0.0, None),
        ((0, -1, 0), 0.0, None), ((0, 0, -1), 0.0, None), ((-1, 0, 0), 0.0, None), ((R2, R2, 0), 0.0, 1e-15)]),
    ("torus", dict(oradius=0.5, iradius=1.0), [  # :813-832
        ((0, 0, 0), -0.5, None), ((1.5, 0, 0), 0.0, None)]),
    ("segment", dict(a=(-1, 0, 0), b=(1, 0, 0)), [  # :834-871
        ((0, 0, 0), -0.1, None), ((-1, 0, 0), -0.1, None), ((1, 0, 0), -0.1, None), ((1, 1.1, 0), 1.0, 1e-15),
        ((0, 1.1, 0), 1.0, 1e-15), ((0, 0, 1.1), 1.0, 1e-15)]),
    ("triprism", dict(h1=1.0, h2=5.0), [  # :873-897
        ((0, 0, 5), 0.0, None), ((0, 1, 0), 0.0, None)]),
    ("capsule", dict(a=(-1, 0, 0), b=(1, 0, 0), r=1.0), [  # :899-929
        ((0, 0, 0), -1.0, None), ((0, 1, 0), 0.0, None), ((2, 0, 0), 0.0, None)]),
    ("plane", dict(a=(0, 0, 1)), [  # :931-965
        ((0, 0, 0), 0.0, None), ((0, 1, 0), 0.0, None), ((2, 0, 0), 0.0, None), ((0, 0, -1), -1.0, None),
        ((0, 0, 1), 1.0, None)]),
    ("cone", dict(a=(0, 0, 0), b=(0, 0, 1), ra=5.0, rb=0.0), [  # :967-993
        ((0, 0, 1), 0.0, None), ((1, 1, 0), 0.0, None)]),
    ("egg", dict(r1=2.5, r2=0.75, h=1.5), [  # :995-1034
        ((0, 0, 0), -2.5, None), ((2.5, 0, 0), 0.0, None), ((0, 2.5 + 1.5, 0), 0.0, 1e-5),
        ((2.5, 2.5, 0), 0.630294, 1e-5)]),
]

# calcNormal on the unit sphere (test/SDF/test_SDF.f90:126-168)
NORMAL_KATS = [((1, 0, 0), (1, 0, 0)), ((0, 1, 0), (0, 1, 0)), ((0, 0, 1), (0, 0, 1))]

# model(sphere .25, box 1) (test/SDF/test_SDF.f90:187-263): (op, point, expected or '>0')
CSG_KATS = [("intersection", (0, 0, 0), -0.25), ("intersection", (0.25, 0, 0), 0.0),
            ("intersection", (0.4, 0, 0), ">0"), ("subtraction", (0, 0, 0), 0.25),
            ("subtraction", (0.25, 0, 0), 0.0)]

# Fresnel (test/fresnel/test_fresnel.f90)
FRESNEL_STAT_TRIALS = 1000000   # :63, :106
FRESNEL_STAT_THR = 5e-4         # :72, :114

# End-to-end (test/end_to_end/test_scat.f90)
SCAT_TEST1_NSCATT = 57.5        # :38
SCAT_TEST1_THR = 0.5
SCAT_TEST2_MOMENTS = [          # :55-63, table 7 of the two-step verification paper
    (0.0, 0.0, 1.0), (0.0, 0.0, 1.9), (0.0, 0.0, 2.71), (0.0, 0.0, 3.349),
    (0.0, 0.0, 2.0), (0.1266666666, 0.1266666666, 5.5466666666), (0.469933, 0.469933, 10.28013),
    (1.091246, 1.091246, 15.91551)]
SCAT_TEST2_THR = (0.1, 0.1, 0.143)  # :69-79

# Philox4x32-10 known-answer vectors (Random123 distribution, kat_vectors)
PHILOX_KATS = [
    ((0, 0), (0, 0, 0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF, 0xFFFFFFFF), (0xFFFFFFFF,) * 4, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0xA4093822, 0x299F31D0), (0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]
