"""B200-native projected-HF grid kernel (energy and orbital gradient over projection grids).

* ``phf_pcc_b200.PHFTools_F.phftools`` -- drop-in for the reference's f2py module
* ``phf_pcc_b200.api``                 -- one-shot calls and reusable GPU plans
* ``phf_pcc_b200.grid`` / ``synth``    -- projection grids and seeded synthetic problems
"""
__version__ = "0.1.0"
