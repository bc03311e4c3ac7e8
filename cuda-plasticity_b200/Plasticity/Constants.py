"""Axis names and the Levi-Civita symbol (reference: Plasticity/Constants.py L1-22)."""
x = 'x'
y = 'y'
z = 'z'
xyz = [x, y, z]

permutation = {(x, y): (1, z), (y, x): (-1, z), (y, z): (1, x), (z, y): (-1, x),
               (x, z): (-1, y), (z, x): (1, y), (x, x): (0., None), (y, y): (0., None),
               (z, z): (0., None)}

perm = {(i, j, k): 0. for i in xyz for j in xyz for k in xyz}
for _i, _j, _k in ((x, y, z), (y, z, x), (z, x, y)):
    perm[_i, _j, _k] = 1.
for _i, _j, _k in ((x, z, y), (z, y, x), (y, x, z)):
    perm[_i, _j, _k] = -1.
