"""Golden constants of the reference's own unit tests (tests.cpp, test.py),
transcribed as data.  They pin the oracle (and through it the CUDA path).
Each block names the tests.cpp / test.py lines it comes from."""
import numpy as np

# tests.cpp:90-96 -- rng(1234) first four xoshiro256** outputs
RNG_1234 = [0x0bab45d9a0e3ae53, 0xd7c640660c19433e, 0xb0dedaa0d09a6691, 0xdec9f41b58ec86eb]

# tests.cpp:146-183 -- multiply_shift draw_one(64, 123456) / draw(1, 64, 123456)
MS_SEED = 123456
MS_A = 2749059519329956733
# tests.cpp:185-222 -- draw(2, 32, 19850)
MS2_SEED = 19850
MS2_A = [3688180003657674949, 11729574476469721337]

# tests.cpp:228-267 -- multiply_add_shift draw_one(128, 123456)
MAS_SEED = 123456
MAS_AB = (2366053268901514180, 2749059519329956733)
# tests.cpp:269-307 -- draw(2, 128, 22201)
MAS2_SEED = 22201
MAS2_AB = [(2016826348251915964, 17696970887482165528), (6666994550483350943, 1097363203091539945)]

# tests.cpp:797-814 -- draw_one(32, 8876) and 100 keys from rng(32149)
MAS3_SEED = 8876
MAS3_AB = (15506110424104283675, 3138147583905456810)
MAS3_KEY_SEED = 32149

# tests.cpp:816-840 -- matmul_sketch<multiply_add_shift>(2, 2, 3483)
SKETCH_SEED = 3483
SKETCH_AB = {
    "h1": [(1312110179027324775, 15465668779316680995), (4555306672462241870, 12288159137770073612)],
    "h2": [(4329212686603688483, 10307990599335447505), (12597734872139453857, 15119207240207437602)],
    "s1": [(11899074044546628492, 298345645907162146), (8628211646415106536, 12647867801867038929)],
    "s2": [(7008367753992221008, 16948937881964684143), (10319872211339334476, 13096518497071785733)],
}

# tests.cpp:312-461 -- tabulation seeds (tables drawn from the same stream)
TAB_SEED_A = 23711   # tab8 m=256, then tab16 with seed+1
TAB_SEED_B = 16321   # draw(2, 128): tab8, then tab16 with seed+1

# tests.cpp:576-615 -- 32-point r2c FFT golden (1e-6 abs), and round trip
FFT_X = np.array([
    0.91527326, 0.07064576, 0.53040597, 0.70546434, 0.36414312, 0.14137265,
    0.50579731, 0.55227775, 0.37729946, 0.95291381, 0.09620142, 0.72017424,
    0.75809317, 0.90013873, 0.46557539, 0.61504573, 0.58568483, 0.25007278,
    0.79962251, 0.22426499, 0.07811993, 0.42820229, 0.72256178, 0.99788856,
    0.1011867, 0.93158399, 0.6872351, 0.95747717, 0.14232377, 0.04623507,
    0.1833904, 0.45529912])
FFT_XHAT = np.array([
    16.2619711 + 0.j, -1.03093929 - 0.05840623j, -1.03078571 + 1.11588142j,
    0.10465414 - 2.23170224j, 1.13343466 - 0.7142413j, 0.89874511 - 0.48200699j,
    0.60648699 - 0.68331135j, 1.02030708 + 2.99294096j, -0.66866564 + 1.50672682j,
    -0.09505786 - 0.3173026j, 1.48484497 + 1.82538006j, 1.3403471 - 0.56288428j,
    0.14009386 - 0.24196106j, -0.0927295 - 0.86637594j, 3.02934147 + 1.79195727j,
    0.49138066 + 0.28645587j, -1.63614286 + 0.j])

# tests.cpp:621-671 -- 32-point natural-order WHT golden (1e-6 abs)
FWHT_X = np.array([
    0.77956498, 0.24374313, 0.66121831, 0.89375154, 0.95073372, 0.11784131,
    0.50483831, 0.44331508, 0.41599355, 0.5194395, 0.26875662, 0.87481817,
    0.9575786, 0.33804587, 0.49530665, 0.73303024, 0.42873154, 0.87784849,
    0.19554847, 0.18266582, 0.78896532, 0.05496766, 0.40847289, 0.30497385,
    0.67434276, 0.70394152, 0.45398693, 0.02708591, 0.01455404, 0.69647227,
    0.69386635, 0.45950925])
FWHT_XHAT = np.array([
    1.61639087e+01, 1.22100944e+00, 9.61619873e-01, 1.69532008e+00,
    2.38965842e-01, -2.11131125e+00, 1.20992754e+00, -9.90377533e-01,
    -4.89547794e-01, 1.97692390e+00, 3.33603927e-01, 1.72112646e+00,
    1.13896243e+00, -1.61840476e+00, -9.18335302e-01, -1.20064715e+00,
    2.23204248e+00, 5.19002383e-01, -2.06580837e+00, 4.10387227e+00,
    -5.77377406e-03, -1.25357604e+00, -3.06495295e+00, 2.75067875e-01,
    4.73622156e-01, 1.07388134e+00, -8.74375765e-01, -1.36142179e+00,
    8.74043671e-01, 2.61878400e+00, 1.65027151e-01, 1.90390037e+00])

# tests.cpp:20-88 -- the small exact matrices (AT is A transposed, row-major)
AT_4x4 = np.array([[1, 5, 9, 13], [2, 6, 10, 14], [3, 7, 11, 15], [4, 8, 12, 16]], dtype=np.float64)
AT_2x4 = np.array([[1, 3, 5, 7], [2, 4, 6, 8]], dtype=np.float64)
AT_4x2 = np.array([[1, 5], [2, 6], [3, 7], [4, 8]], dtype=np.float64)
B_4x4 = np.arange(17, 33, dtype=np.float64).reshape(4, 4)
B_2x4 = np.arange(9, 17, dtype=np.float64).reshape(2, 4)
B_4x2 = np.arange(9, 17, dtype=np.float64).reshape(4, 2)
B_4x8 = np.arange(1, 33, dtype=np.float64).reshape(4, 8)
C_4x4x4 = np.array([[250, 260, 270, 280], [618, 644, 670, 696], [986, 1028, 1070, 1112],
                    [1354, 1412, 1470, 1528]], dtype=np.float64)
C_4x2x4 = np.array([[35, 38, 41, 44], [79, 86, 93, 100], [123, 134, 145, 156],
                    [167, 182, 197, 212]], dtype=np.float64)
C_2x4x2 = np.array([[130, 140], [322, 348]], dtype=np.float64)
C_2x4x8 = np.array([[170, 180, 190, 200, 210, 220, 230, 240],
                    [378, 404, 430, 456, 482, 508, 534, 560]], dtype=np.float64)
# (AT, B, C, n_a, n_inner, n_b) as used by tests.cpp:906-941 / 1114-1149
SMALL_PRODUCTS = [
    (AT_4x4, B_4x4, C_4x4x4),
    (AT_2x4, B_2x4, C_4x2x4),
    (AT_4x2, B_4x2, C_2x4x2),
    (AT_4x2, B_4x8, C_2x4x8),
]
# tests.cpp:842 / 1052 -- (d, b) lists, seed 25926; asserted when d>1 and b>=32
SMALL_DB_FFT = [(1, 2), (1, 8), (1, 32), (3, 2), (3, 8), (5, 32)]
SMALL_DB_FWHT = [(1, 2), (1, 8), (1, 32), (3, 2), (3, 8), (7, 32)]
SMALL_SEED = 25926

# tests.cpp:944-1003 / 1152-1211 -- 16x16 drng(15954) vs dgemm at 1e-12
RAND16_SEED = 15954
RAND16_FFT = [("multiply add shift", 5, 1024, 1), ("multiply shift", 5, 1024, 2),
              ("tabulation8", 11, 2048, 3), ("tabulation16", 11, 1024, 4)]
RAND16_FWHT = [("multiply add shift", 5, 2048, 1), ("multiply shift", 5, 2048, 2),
               ("tabulation8", 11, 2048, 3), ("tabulation16", 11, 1024, 4)]

# test.py:30-48 -- the Python test's fixtures (note B_4x8 = arange(9, 41))
PY_AT_4x4 = np.ascontiguousarray(np.arange(1, 17, dtype=np.float64).reshape(4, 4).T)
PY_B_4x4 = np.arange(17, 33, dtype=np.float64).reshape(4, 4)
PY_AT_2x4 = np.ascontiguousarray(np.arange(1, 9, dtype=np.float64).reshape(4, 2).T)
PY_B_2x4 = np.arange(9, 17, dtype=np.float64).reshape(2, 4)
PY_AT_4x2 = np.ascontiguousarray(np.arange(1, 9, dtype=np.float64).reshape(2, 4).T)
PY_B_4x2 = np.arange(9, 17, dtype=np.float64).reshape(4, 2)
PY_B_4x8 = np.arange(9, 41, dtype=np.float64).reshape(4, 8)
PY_SEED = 13794
# test.py:53-64
PY_PARAMS_SMALL = {
    ("fft", None): (1, 256), ("fft", "multiply shift"): (1, 128),
    ("fft", "multiply add shift"): (1, 256), ("fft", "tabulation8"): (1, 128),
    ("fft", "tabulation16"): (1, 64), ("fwht", None): (1, 32),
    ("fwht", "multiply shift"): (1, 64), ("fwht", "multiply add shift"): (1, 32),
    ("fwht", "tabulation8"): (1, 64), ("fwht", "tabulation16"): (1, 64),
}
# test.py:90-91
PY_SEED1, PY_SEED2 = 27548, 23340
# test.py:122-133 and the 16x16 integer matrices of default_rng(27840)
PY_PARAMS_16 = {
    ("fft", None): (7, 1024), ("fft", "multiply shift"): (5, 1024),
    ("fft", "multiply add shift"): (7, 1024), ("fft", "tabulation8"): (9, 2048),
    ("fft", "tabulation16"): (9, 1024), ("fwht", None): (11, 1024),
    ("fwht", "multiply shift"): (9, 1024), ("fwht", "multiply add shift"): (11, 1024),
    ("fwht", "tabulation8"): (9, 1024), ("fwht", "tabulation16"): (11, 2048),
}
PY_RNG16_SEED = 27840


def py_fixtures():
    """test.py:65-67 pairs (AT, B, C)."""
    return [(PY_AT_4x4, PY_B_4x4, PY_AT_4x4.T @ PY_B_4x4),
            (PY_AT_4x2, PY_B_4x2, PY_AT_4x2.T @ PY_B_4x2),
            (PY_AT_2x4, PY_B_2x4, PY_AT_2x4.T @ PY_B_2x4),
            (PY_AT_4x2, PY_B_4x8, PY_AT_4x2.T @ PY_B_4x8)]


def py_int16():
    """test.py:135-139: integer 16x16 A, B from default_rng(27840)."""
    rng = np.random.default_rng(PY_RNG16_SEED)
    A = rng.integers(-10, 11, (16, 16)).astype(np.float64)
    B = rng.integers(-10, 11, (16, 16)).astype(np.float64)
    return np.ascontiguousarray(A.T), B, A @ B
