"""Write triangle arrays as a Wavefront OBJ + MTL pair that the reference's
loader semantics read back to the same arrays (tests only)."""
from __future__ import annotations

import os

import numpy as np

# reference Material enum -> a usemtl name that maps to it (src/ObjLoader.cpp:51-73)
SPECIAL = {1: "Mirror", 2: "Glass", 3: "Marble", 4: "Bumpy", 5: "Parallax", 6: "Metal", 7: "Dispersive",
           8: "Wax", 9: "NormalMap", 10: "Emissive"}


def write_obj(directory: str, stem: str, v9: np.ndarray, rgb: np.ndarray, material: np.ndarray,
              share_vertices: bool = False) -> str:
    """Vertices are written with 9 significant digits (exact float round trip)
    and loaded at scale 1; Kd = (rgb + 0.5) / 255 so int(Kd * 255) == rgb.
    With share_vertices, corners at bit-identical positions share one ``v`` line
    (so the loader's vertex-normal smoothing sees the mesh's connectivity)."""
    names = {}
    mtl_lines = []
    faces_by = []
    for i in range(v9.shape[0]):
        m = int(material[i])
        col = tuple(int(c) for c in rgb[i])
        if m == 0:
            name = "D_%d_%d_%d" % col
        else:
            name = SPECIAL[m]
            if name in names and names[name] != col:
                raise ValueError(f"material {name} used with two colours")
        if name not in names:
            names[name] = col
            kd = " ".join("%.9g" % ((c + 0.5) / 255.0) for c in col)
            mtl_lines.append(f"newmtl {name}\nKd {kd}\n")
        faces_by.append(name)
    with open(os.path.join(directory, stem + ".mtl"), "w") as f:
        f.write("\n".join(mtl_lines))
    lines = [f"mtllib {stem}.mtl"]
    v9 = np.asarray(v9, np.float32)
    if share_vertices:
        index = {}
        for i in range(v9.shape[0]):
            for k in range(3):
                key = v9[i, 3 * k:3 * k + 3].tobytes()
                if key not in index:
                    index[key] = len(index) + 1
                    x, y, z = (float(c) for c in v9[i, 3 * k:3 * k + 3])
                    lines.append("v %.9g %.9g %.9g" % (x, y, z))
    current = None
    for i in range(v9.shape[0]):
        if faces_by[i] != current:
            current = faces_by[i]
            lines.append(f"usemtl {current}")
        if share_vertices:
            ids = [index[v9[i, 3 * k:3 * k + 3].tobytes()] for k in range(3)]
            lines.append(f"f {ids[0]}/ {ids[1]}/ {ids[2]}/")
            continue
        for k in range(3):
            x, y, z = (float(c) for c in v9[i, 3 * k:3 * k + 3])
            lines.append("v %.9g %.9g %.9g" % (x, y, z))
        b = 3 * i + 1
        lines.append(f"f {b}/ {b + 1}/ {b + 2}/")
    path = os.path.join(directory, stem + ".obj")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path
