"""The settings record's JSON number format and hash (host code in
csrc/config.cpp), compiled here with a small driver, no GPU needed.

Floats are written as the reference's serializer writes an f32 (the
shortest digits that round-trip, positional for decimal exponents from -5
to 13, else d.ddde<exp>); the checks are hand-worked values and numpy's
shortest f32 digits over a seeded sample.  The hash is 64-bit FNV-1a
(crates/cloth_core/src/config.rs:205-214)."""
import os
import subprocess

import numpy as np
import pytest

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "taremincloth_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "config.hpp"
int main(int argc, char** argv) {
  if (argc > 1 && std::strcmp(argv[1], "hash") == 0) {
    std::printf("%llu\n", (unsigned long long)tcloth::settings_hash(argv[2]));
    return 0;
  }
  if (argc > 1 && std::strcmp(argv[1], "json") == 0) {
    std::printf("%s\n", tcloth::settings_json(tcloth::SimSettings{}).c_str());
    return 0;
  }
  unsigned bits;
  while (std::scanf("%x", &bits) == 1) {
    float f;
    std::memcpy(&f, &bits, 4);
    std::printf("%s\n", tcloth::json_f32(f).c_str());
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    d = tmp_path_factory.mktemp("cfg")
    src = d / "driver.cpp"
    src.write_text(DRIVER)
    exe = d / "driver"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{CSRC}", str(src), os.path.join(CSRC, "config.cpp"), "-o",
                    str(exe)], check=True)
    return str(exe)


def fmt(driver, values):
    bits = np.asarray(values, np.float32).view(np.uint32)
    out = subprocess.run([driver], input="\n".join(f"{b:x}" for b in bits), capture_output=True, text=True,
                         check=True).stdout.split()
    return out


def layout(x):
    """Positional / exponent layout from numpy's shortest f32 digits."""
    s = np.format_float_scientific(np.float32(x), unique=True, trim="-")
    neg = s.startswith("-")
    s = s.lstrip("-")
    mant, e = s.split("e")
    digits = mant.replace(".", "")
    kk = int(e) + 1
    k = kk - len(digits)
    if k >= 0 and kk <= 13:
        t = digits + "0" * k + ".0"
    elif 0 < kk <= 13:
        t = digits[:kk] + "." + digits[kk:]
    elif -6 < kk <= 0:
        t = "0." + "0" * (-kk) + digits
    elif len(digits) == 1:
        t = f"{digits}e{kk - 1}"
    else:
        t = f"{digits[0]}.{digits[1:]}e{kk - 1}"
    return ("-" if neg else "") + t


def test_hand_worked_values(driver):
    cases = {9.81: "9.81", -9.81: "-9.81", 0.0: "0.0", 1.0: "1.0", 0.005: "0.005", 1e-9: "1e-9",
             1.5e-10: "1.5e-10", 10000.0: "10000.0", 1e12: "1000000000000.0", 1e13: "1e13", 1e-6: "0.000001",
             1e-7: "1e-7", 123456.79: "123456.79", 3.4028235e38: "3.4028235e38", 0.1: "0.1", 1.3: "1.3",
             0.008: "0.008", 600.0: "600.0"}
    got = fmt(driver, list(cases))
    assert got == list(cases.values())
    assert fmt(driver, [np.inf, np.nan]) == ["null", "null"]


def test_shortest_digits_sample(driver):
    rng = np.random.default_rng(7)
    x = np.concatenate([rng.uniform(-1e4, 1e4, 300), 10.0 ** rng.uniform(-12, 20, 300),
                        rng.integers(-10 ** 6, 10 ** 6, 100).astype(np.float64)]).astype(np.float32)
    got = fmt(driver, x)
    assert got == [layout(v) for v in x]
    # every text parses back to the same f32
    assert (np.array([float(t) for t in got], np.float32).view(np.uint32) == x.view(np.uint32)).all()


def test_hash_is_fnv1a(driver):
    def fnv(s):
        h = 0xcbf29ce484222325
        for b in s.encode():
            h = ((h ^ b) * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
        return h
    for s in ("", "a", '{"version":1}'):
        out = subprocess.run([driver, "hash", s], capture_output=True, text=True, check=True).stdout
        assert int(out) == fnv(s)


def test_record_field_order(driver):
    import json
    from taremincloth_b200.simulator import CONFIG_DEFAULTS
    out = subprocess.run([driver, "json"], capture_output=True, text=True, check=True).stdout.strip()
    d = json.loads(out)
    assert list(d) == list(CONFIG_DEFAULTS)
    assert " " not in out
