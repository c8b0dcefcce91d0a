"""Regenerates h2_air_9sp.json: the species/reaction tables of the 9-species,
19-reaction H2-air CHEMKIN mechanism (combustion_mechanism.inp + therm.dat +
tran.dat of the reference's input_files/chemistry), parsed by chemdata.py;
and h2_mixing_4sp.json: the species tables of the non-reacting set of
H2_mech_mixing.inp (the reference reads no reactions for it, reaction = 0).

usage: python make_mechanism.py <dir holding the three CHEMKIN files>
"""
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))

import chemdata  # noqa: E402

src = Path(sys.argv[1])
mech = chemdata.load_chemkin(src / "combustion_mechanism.inp", src / "therm.dat", src / "tran.dat")
chemdata.save_json(mech, HERE / "h2_air_9sp.json")
print(mech.names, mech.n_reac)
mix = chemdata.load_chemkin(src / "H2_mech_mixing.inp", src / "therm.dat", src / "tran.dat", reactions=False)
chemdata.save_json(mix, HERE / "h2_mixing_4sp.json")
print(mix.names, mix.n_reac)
