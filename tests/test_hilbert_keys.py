"""The property the simulation's Hilbert-ordered octree relies on (csrc/sort.cu, hilbert_from_axes):
J. Skilling's transform of the integer coordinates that the octant digits spell gives a key whose
first 3d bits name exactly one level-d cube, every one of the 8^d cubes once, so sorting by it keeps
every octree node's particles contiguous. Checked on a restatement of the kernel's branch-free
transform (the GPU tests check the tree built from it against the oracle)."""
from collections import defaultdict


def hilbert_from_axes(x0, x1, x2, bits):
    X = [x0, x1, x2]
    for b in range(bits - 1, 0, -1):
        q = 1 << b
        p = q - 1
        for i in range(3):
            t = (X[0] ^ X[i]) & p
            inv = (X[i] & q) != 0
            X[0] ^= p if inv else t
            if i:
                X[i] ^= 0 if inv else t
    X[1] ^= X[0]
    X[2] ^= X[1]
    t = 0
    for b in range(bits - 1, 0, -1):
        if X[2] & (1 << b):
            t ^= (1 << b) - 1
    X = [x ^ t for x in X]
    key = 0
    for j in range(bits - 1, -1, -1):
        key = (key << 3) | (((X[0] >> j) & 1) << 2) | (((X[1] >> j) & 1) << 1) | ((X[2] >> j) & 1)
    return key


def test_key_prefixes_name_the_octant_cubes():
    bits = 4
    n = 1 << bits
    keys = {}
    for x in range(n):
        for y in range(n):
            for z in range(n):
                keys[(x, y, z)] = hilbert_from_axes(x, y, z, bits)
    assert sorted(keys.values()) == list(range(n ** 3))  # a bijection onto 0 .. 8^bits - 1
    for d in range(1, bits + 1):
        cubes = defaultdict(set)
        for (x, y, z), k in keys.items():
            cubes[k >> (3 * (bits - d))].add((x >> (bits - d), y >> (bits - d), z >> (bits - d)))
        assert len(cubes) == 8 ** d and all(len(c) == 1 for c in cubes.values()), d


def test_consecutive_keys_are_face_neighbours():
    """A Hilbert curve: consecutive keys are adjacent cells (one unit step along one axis)."""
    bits = 3
    n = 1 << bits
    cell = {hilbert_from_axes(x, y, z, bits): (x, y, z) for x in range(n) for y in range(n) for z in range(n)}
    for k in range(n ** 3 - 1):
        a, b = cell[k], cell[k + 1]
        assert sum(abs(u - v) for u, v in zip(a, b)) == 1, (k, a, b)


def test_state_machine_keys_match_the_transform():
    """The device computes the Hilbert keys digit by digit with a state machine derived on the host
    from the transform (csrc/sort.cu, derive_hilbert_fsm); the library's self-check compares the two
    on random coordinates at both key depths (21 digits; 19 under a batch of boxes)."""
    import ctypes as C
    import importlib
    native = importlib.import_module("cosmological-particle-simulation_b200._native")
    for levels in (21, 19):
        bad, states = C.c_uint64(), C.c_int()
        assert native.lib().cpm_hilbert_fsm_check(levels, 200000, 12345, C.byref(bad), C.byref(states)) == 0
        assert states.value in (12, 24), (levels, states.value)
        assert bad.value == 0, (levels, bad.value)


def test_state_machine_check_rejects_other_depths():
    import ctypes as C
    import importlib
    native = importlib.import_module("cosmological-particle-simulation_b200._native")
    bad, states = C.c_uint64(), C.c_int()
    for levels in (0, 20, 22):
        assert native.lib().cpm_hilbert_fsm_check(levels, 10, 1, C.byref(bad), C.byref(states)) != 0
