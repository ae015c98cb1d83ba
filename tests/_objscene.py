"""Writes OBJ / MTL test scenes (this project's own content): a Cornell-style
box of quads with corner normals and an emissive ceiling quad, plus two
blocks, and small files exercising every face form the reader accepts."""
import os

MTL = """# materials of the test box
newmtl white
Kd 0.725 0.71 0.68
Ke 0 0 0
newmtl red
Kd 0.63 0.065 0.05
newmtl green
Kd 0.14 0.45 0.091
newmtl lamp
Kd 0.78 0.78 0.78
Ke 17 12 4
"""


def _quad(lines, verts, normal, vbase, nbase):
    for v in verts:
        lines.append("v %.6f %.6f %.6f" % v)
    lines.append("vn %.6f %.6f %.6f" % normal)
    n = nbase + 1
    lines.append("f %d//%d %d//%d %d//%d %d//%d" % (vbase + 1, n, vbase + 2, n, vbase + 3, n, vbase + 4, n))
    return vbase + 4, nbase + 1


def _block(lines, cx, cz, hx, hz, height, angle, vb, nb):
    import math
    c, s = math.cos(angle), math.sin(angle)
    def p(x, y, z):
        return (cx + c * x - s * z, y, cz + s * x + c * z)
    x0, x1, z0, z1 = -hx, hx, -hz, hz
    faces = [([p(x0, height, z0), p(x0, height, z1), p(x1, height, z1), p(x1, height, z0)], (0, 1, 0)),
             ([p(x0, 0, z1), p(x1, 0, z1), p(x1, height, z1), p(x0, height, z1)], (s * 0 + -s, 0, c)),
             ([p(x1, 0, z0), p(x0, 0, z0), p(x0, height, z0), p(x1, height, z0)], (s, 0, -c)),
             ([p(x1, 0, z1), p(x1, 0, z0), p(x1, height, z0), p(x1, height, z1)], (c, 0, s)),
             ([p(x0, 0, z0), p(x0, 0, z1), p(x0, height, z1), p(x0, height, z0)], (-c, 0, -s))]
    for verts, n in faces:
        vb, nb = _quad(lines, verts, n, vb, nb)
    return vb, nb


def write_cornell(directory, name="box"):
    """A 2 x 2 x 2 box (y up, opening towards +z), red left / green right
    walls, a lamp under the ceiling and two rotated blocks. Returns the OBJ path."""
    lines = ["# test box", "mtllib %s.mtl" % name]
    vb = nb = 0
    walls = [("white", [(-1, 0, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1)], (0, 1, 0)),
             ("white", [(-1, 2, 1), (-1, 2, -1), (1, 2, -1), (1, 2, 1)], (0, -1, 0)),
             ("white", [(-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1)], (0, 0, 1)),
             ("red", [(-1, 0, 1), (-1, 0, -1), (-1, 2, -1), (-1, 2, 1)], (1, 0, 0)),
             ("green", [(1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1)], (-1, 0, 0)),
             ("lamp", [(-0.25, 1.98, -0.25), (0.25, 1.98, -0.25), (0.25, 1.98, 0.25), (-0.25, 1.98, 0.25)],
              (0, -1, 0))]
    for mat, verts, n in walls:
        lines.append("usemtl " + mat)
        vb, nb = _quad(lines, verts, n, vb, nb)
    lines.append("usemtl white")
    vb, nb = _block(lines, -0.35, -0.3, 0.3, 0.3, 1.2, 0.3, vb, nb)
    vb, nb = _block(lines, 0.35, 0.35, 0.3, 0.3, 0.6, -0.3, vb, nb)
    with open(os.path.join(directory, name + ".mtl"), "w") as f:
        f.write(MTL)
    path = os.path.join(directory, name + ".obj")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path
