"""Generates tests/golden/known_answers.json.

The known answers of AdaptiveCpp's own tests for the data-parallel primitive
path, re-expressed as (inputs-recipe, expected value) pairs.  Each expected
value is recomputed here with plain Python integers/floats in the serial
std:: order the reference tests compare against; nothing is copied from the
test sources except the recipes (sizes, generators, init values, predicates).

Sources (AdaptiveCpp tree):
  tests/pstl/reduce.cpp:24-86            data[i] = i, sizes 0/1/127/1000/10^6
  tests/pstl/transform_reduce.cpp:25-154 same, identity transform
  tests/pstl/inclusive_scan.cpp:71-195   data[i] = i, plus / multiply, init 3
  tests/pstl/exclusive_scan.cpp:88-190   same structure
  tests/pstl/copy_if.cpp:24-64           predicate x % 2 == 0, none/all/half
  tests/sycl/reduction.cpp:25-378        plus/multiplies generators, sizes
  tests/sycl/atomic.cpp:81-125           2048 work-items fetch_add(-i)
Also pins the first values of the synthetic-input generator (SplitMix64 /
Box-Muller), restated independently in Python below.

Run:  python tests/golden/make_golden.py
"""
import json
import math
import os

M64 = (1 << 64) - 1


def wrap(v, bits, signed):
    v &= (1 << bits) - 1
    if signed and v >= 1 << (bits - 1):
        v -= 1 << bits
    return v


def pstl_reduce_cases():
    out = []
    for n, init, bits in [(0, 10, 32), (1, 10, 32), (127, 10, 32), (1000, 0, 32), (1000000, 0, 64)]:
        out.append({"n": n, "init": init, "bits": bits,
                    "expected": wrap(init + n * (n - 1) // 2, bits, True),
                    "expected_noinit": wrap(n * (n - 1) // 2, bits, True)})
    return out


def scan_cases():
    out = []
    for n in [0, 1, 127, 1000, 1048576]:
        # plus, init 3 ; int data[i] = i  (int32 arithmetic, wraps)
        incl, acc, acc_i = [], 0, 3
        s_plain = s_init = 0
        last_plain = last_init = None
        excl_last = None
        excl_sum = 0
        e = 3
        for i in range(n):
            acc = wrap(acc + i, 32, True)
            acc_i = wrap(acc_i + i, 32, True)
            s_plain = (s_plain + acc) & M64
            s_init = (s_init + acc_i) & M64
            last_plain, last_init = acc, acc_i
            excl_sum = (excl_sum + e) & M64
            excl_last = e
            e = wrap(e + i, 32, True)
        out.append({"n": n, "op": "plus", "init": 3,
                    "incl_last": last_plain, "incl_sum_mod64": s_plain,
                    "incl_init_last": last_init, "incl_init_sum_mod64": s_init,
                    "excl_last": excl_last, "excl_sum_mod64": excl_sum})
        # multiply with init 3: data[0] = 0 makes every inclusive value 0;
        # exclusive: first value 3, then 0.
        out.append({"n": n, "op": "multiplies", "init": 3,
                    "incl_all_zero": True, "excl_first": 3 if n else None,
                    "excl_rest_zero": True})
    return out


def copy_if_cases():
    out = []
    for name, n, gen in [("empty", 0, "i"), ("single", 1, "i+3"), ("none", 1000, "1"),
                         ("all", 1000, "2i"), ("half", 1000, "i")]:
        data = [eval(gen.replace("2i", "2*i"), {"i": i}) for i in range(n)]
        kept = [x for x in data if x % 2 == 0]
        out.append({"case": name, "n": n, "gen": gen, "count": len(kept),
                    "kept_sum": sum(kept), "kept_first": kept[:3]})
    return out


def sycl_reduction_cases():
    def plus_gen(i):
        return i

    def mul_gen(i):
        if i > 1500:
            return 1
        return 2 if i % 100 == 0 else 1

    out = []
    for n in [128, 128 * 128, 64 * 64 * 64, 1000, 20]:
        for T, bits, signed in [("int32", 32, True), ("uint32", 32, False), ("int64", 64, True)]:
            s = wrap(sum(plus_gen(i) for i in range(n)), bits, signed)
            p = 1
            for i in range(n):
                p = wrap(p * mul_gen(i), bits, signed)
            out.append({"n": n, "type": T, "plus": s, "multiplies": p})
        fs = float(sum(plus_gen(i) for i in range(n)))
        fp = float(math.prod(mul_gen(i) for i in range(n)))
        out.append({"n": n, "type": "float", "plus": fs, "multiplies": fp, "rel_tol": 1e-3})
    out.append({"n": 1024, "type": "int32", "iota_sum": 523776, "iota_max": 1023})
    return out


def atomic_cases():
    # 2048 work-items, acc[0] starts at init(0) = 0, items 1..2047 add init(i) = -i
    return [{"n": 2048, "fetch_add_expected": sum(-i for i in range(1, 2048))}]


# ---- independent restatement of the synthetic generator (b2p_synth_fill)
def mix(seed, i, stream):
    z = (seed * 0x9E3779B97F4A7C15 + (i + 1) * 0xD1B54A32D192ED03 + (stream + 1) * 0x8CB92BA72F3D8DD7) & M64
    z = (z + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def unif(seed, i, s):
    return ((mix(seed, i, s) >> 11) + 1) * 2.0 ** -53


def normal(seed, i, s0):
    return math.sqrt(-2.0 * math.log(unif(seed, i, s0))) * math.cos(6.283185307179586 * unif(seed, i, s0 + 1))


def synth_pins():
    import struct

    def f32(x):
        return struct.unpack("f", struct.pack("f", x))[0]

    ints = [-1000 + mix(0, i, 0) % 2001 for i in range(16)]
    normals = []
    for i in range(16):
        if unif(1, i, 3) <= 0.125:
            normals.append(f32(1e-6 * normal(1, i, 4)))
        else:
            normals.append(f32(normal(1, i, 1)))
    u32 = [mix(4, i, 0) >> 32 for i in range(16)]
    return {"int32_seed0": ints, "fp32_seed1_frac0.125": normals, "uint32_seed4": u32}


def main():
    doc = {
        "pstl_reduce": pstl_reduce_cases(),
        "pstl_scan": scan_cases(),
        "pstl_copy_if": copy_if_cases(),
        "sycl_reduction": sycl_reduction_cases(),
        "atomic": atomic_cases(),
        "synth": synth_pins(),
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_answers.json")
    with open(path, "w") as f:
        json.dump(doc, f, indent=1)
    print(path)


if __name__ == "__main__":
    main()
