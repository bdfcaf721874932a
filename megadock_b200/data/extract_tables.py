"""Regenerate the data assets in this directory from MEGADOCK's parameter tables.

MEGADOCK keeps its force-field tables and rotation sets as C++ initialisers
(src/parameter.cpp) and its FFT-size tables in src/control.cpp.  A drop-in
replacement must use exactly the same numbers, so this script extracts them
mechanically (no hand copying) into plain data files:

  charmm_radius.tsv  key<TAB>value   Parameter::charmm_radius  (parameter.cpp:473-1391)
  charmm_charge.tsv  key<TAB>value   Parameter::charmm_charge  (parameter.cpp:1394-2312)
  ace.tsv            key<TAB>value   Parameter::ace_value      (parameter.cpp:2315-3790)
  rotations_<n>.f32  float32[n*3]    Parameter::dangle_rot<n>  (parameter.cpp:3793-61887)
  fft_tables.tsv     set<TAB>sizes   Control::gridtable_*      (control.cpp:91-282)

Values keep the reference's conversion chain: a decimal literal is a C double
converted to float, which is what ``np.float32(float(text))`` does.  The table
files keep the decimal text; their readers convert the same way.  Where a key
occurs more than once, the first occurrence wins (std::map::insert semantics).

Usage:  python extract_tables.py <path to the MEGADOCK src directory>
"""
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

_INSERT = re.compile(r'(_Charmmr|_Charmmc|_ACE)\.insert\(map<string,float>::value_type\("([^"]*)",\s*([-+0-9.eE]+)\)\)')
_FUNC = re.compile(r'^void Parameter::(\w+)\(\)')
_GRID_FUNC = re.compile(r'^void Control::gridtable_(\w+)\(')
_GRID_SET = {"13base_normal": 13, "07base_normal": 7, "11base_normal": 11,
             "fftw_custom": 0, "cufft_custom": 1}


def _strip_comments(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def extract_atom_tables(parameter_cpp):
    tables = {"_Charmmr": {}, "_Charmmc": {}, "_ACE": {}}
    for m in _INSERT.finditer(_strip_comments(parameter_cpp)):
        name, key, val = m.groups()
        tables[name].setdefault(key, val)
    return tables


def extract_rotations(parameter_cpp):
    """Return {n: float32 array (n,3)} for every dangle_rot<n> function."""
    out = {}
    lines = parameter_cpp.split("\n")
    i = 0
    while i < len(lines):
        m = _FUNC.match(lines[i])
        if m and m.group(1).startswith("dangle_rot"):
            # collect the body up to the closing brace of the initialiser
            body = []
            j = i + 1
            while "};" not in lines[j]:
                body.append(lines[j])
                j += 1
            text = _strip_comments("\n".join(body))
            start = text.index("{", text.index("Zangle[]"))
            nums = re.findall(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?", text[start:])
            vals = np.array([np.float32(float(v)) for v in nums], dtype=np.float32)
            assert vals.size % 3 == 0, m.group(1)
            out[vals.size // 3] = vals.reshape(-1, 3)
            i = j
        i += 1
    return out


def extract_fft_tables(control_cpp):
    out = {}
    lines = _strip_comments(control_cpp).split("\n")
    i = 0
    while i < len(lines):
        m = _GRID_FUNC.match(lines[i])
        if m and m.group(1) in _GRID_SET:
            j = i
            while "grid_table[]" not in lines[j]:
                j += 1
            body = []
            while True:
                body.append(lines[j])
                if "};" in lines[j]:
                    break
                j += 1
            text = "\n".join(body)
            text = text[text.index("{") + 1:text.index("}")]
            out[_GRID_SET[m.group(1)]] = [int(v) for v in re.findall(r"\d+", text)]
            i = j
        i += 1
    return out


def main(src):
    src = Path(src)
    param = (src / "parameter.cpp").read_text(errors="replace")
    control = (src / "control.cpp").read_text(errors="replace")
    names = {"_Charmmr": "charmm_radius.tsv", "_Charmmc": "charmm_charge.tsv", "_ACE": "ace.tsv"}
    for name, tab in extract_atom_tables(param).items():
        with open(HERE / names[name], "w") as f:
            for k, v in tab.items():
                f.write(f"{k}\t{v}\n")
    for n, arr in extract_rotations(param).items():
        arr.astype("<f4").tofile(HERE / f"rotations_{n}.f32")
    with open(HERE / "fft_tables.tsv", "w") as f:
        for k, v in sorted(extract_fft_tables(control).items()):
            f.write(f"{k}\t{' '.join(map(str, v))}\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python extract_tables.py <MEGADOCK src directory>")
    main(sys.argv[1])
