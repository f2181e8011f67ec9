"""Writes compress_trivial_n6-6_l5.txt: the compress file that the reference's
own generator (tools/compress_indices/compress_indices.py, mode "trivial", as
shipped: n_max [6, 6], l_max 5) prints. Run where the reference tree is present,
with the root of that tree as the one argument:

    python tests/golden/make_compress_trivial.py <reference tree>
"""
import pathlib
import subprocess
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_compress_trivial.py <root of the reference tree>")
ref = pathlib.Path(sys.argv[1])
out = subprocess.run([sys.executable, str(ref / "tools" / "compress_indices" / "compress_indices.py")],
                     check=True, capture_output=True, text=True).stdout
(pathlib.Path(__file__).parent / "compress_trivial_n6-6_l5.txt").write_text(out)
