"""Writes tests/golden/csf_argon.npz: the reference's argon electron cross sections (its
csf/Ar.txt, elastic, and csf/Ar+.txt, ionisation from 15.76 eV), read with
pic_cuda_b200.xs.read_cross_section (the semantics of mcc.cu:17-41), so that tests can feed
the real non-uniform tables to the engine where the reference tree is absent.

    python tests/golden/make_csf_fixture.py [reference_root] [outdir]
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from pic_cuda_b200.xs import read_cross_section  # noqa: E402


def main(ref: Path, out: Path):
    e_el, s_el = read_cross_section(ref / "csf" / "Ar.txt")
    e_iz, s_iz = read_cross_section(ref / "csf" / "Ar+.txt")
    assert e_el and e_iz, "cross-section files not found under " + str(ref)
    np.savez_compressed(out / "csf_argon.npz", elastic_E=np.array(e_el), elastic_sigma=np.array(s_el),
                        ionization_E=np.array(e_iz), ionization_sigma=np.array(s_iz))
    print("wrote", out / "csf_argon.npz", len(e_el), len(e_iz))


if __name__ == "__main__":
    ref = Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference")
    out = Path(sys.argv[2]) if len(sys.argv) > 2 else Path(__file__).resolve().parent
    main(ref, out)
