"""Generate the D3Q19 MRT moment basis used by the oracle harness.

Test infrastructure only.  The reference ships MRT matrix data for D2Q9 only
(src/lbm/collisionMRT.h:55-91); its generic MRT algorithm
(src/lbm/collisionMRT.h:132-190) is lattice-independent.  This script writes
the Gram-Schmidt D3Q19 basis of d'Humieres, Ginzburg, Krafczyk, Lallemand and
Luo, Phil. Trans. R. Soc. A 360 (2002) 437-451, evaluated on the reference's
D3Q19 velocity ordering (src/lbm/lattice_set.h:263-266), as explicit
specialisations of the reference's ``mrtdata`` variable templates, so that the
oracle harness can run the reference's own generic MRT collision on D3Q19.

Run:  python oracle/gen_mrt_d3q19.py > oracle/mrt_d3q19_table.h
"""
from fractions import Fraction
import math

# D3Q19 velocities in the reference ordering (src/lbm/lattice_set.h:263-266).
C = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
     (1, 1, 0), (-1, -1, 0), (1, 0, 1), (-1, 0, -1), (0, 1, 1), (0, -1, -1), (1, -1, 0),
     (-1, 1, 0), (1, 0, -1), (-1, 0, 1), (0, 1, -1), (0, -1, 1)]


def basis_row(k, c):
    """Row k of the d'Humieres 2002 moment basis evaluated at velocity c."""
    x, y, z = c
    c2 = x * x + y * y + z * z
    rows = [
        1,                                   # rho
        19 * c2 - 30,                        # e
        (21 * c2 * c2 - 53 * c2 + 24) // 2,  # epsilon
        x, (5 * c2 - 9) * x,                 # j_x, q_x
        y, (5 * c2 - 9) * y,                 # j_y, q_y
        z, (5 * c2 - 9) * z,                 # j_z, q_z
        3 * x * x - c2,                      # 3 p_xx
        (3 * c2 - 5) * (3 * x * x - c2),     # 3 pi_xx
        y * y - z * z,                       # p_ww
        (3 * c2 - 5) * (y * y - z * z),      # pi_ww
        x * y, y * z, x * z,                 # p_xy, p_yz, p_xz
        x * (y * y - z * z),                 # m_x
        y * (z * z - x * x),                 # m_y
        z * (x * x - y * y),                 # m_z
    ]
    return rows[k]


M = [[basis_row(k, c) for c in C] for k in range(19)]
NORM = [sum(v * v for v in row) for row in M]
# shear-viscosity moments relax with omega = 1/tau; conserved moments with 0.
SHEAR = [9, 11, 13, 14, 15]
CONSERVED = [0, 3, 5, 7]


def check():
    for a in range(19):
        for b in range(19):
            dot = sum(M[a][i] * M[b][i] for i in range(19))
            assert (dot == 0) == (a != b), (a, b, dot)


def main():
    check()
    out = []
    out.append("// Generated by oracle/gen_mrt_d3q19.py -- do not edit.")
    out.append("// D3Q19 Gram-Schmidt MRT basis (d'Humieres et al. 2002) on the reference's")
    out.append("// velocity ordering, as specialisations of the reference's mrtdata templates.")
    out.append("#pragma once")
    out.append("namespace mrtdata {")
    out.append("template <>")
    out.append("__constexpr__ Fraction<> M<3, 19>[19][19] = {")
    for row in M:
        out.append("  {" + ", ".join(f"{v:3d}" for v in row) + "},")
    out.append("};")
    out.append("template <>")
    out.append("__constexpr__ Fraction<> InvM<3, 19>[19][19] = {")
    for i in range(19):
        ent = []
        for j in range(19):
            fr = Fraction(M[j][i], NORM[j])
            ent.append(f"{{{fr.numerator}, {fr.denominator}}}")
        out.append("  {" + ", ".join(ent) + "},")
    out.append("};")
    out.append("template <>")
    svals = []
    for k in range(19):
        if k in CONSERVED:
            svals.append("0")
        elif k in SHEAR:
            svals.append("1")  # overwritten by omega in MRT_Feq_RhoU
        else:
            svals.append("{6, 5}")
    out.append("__constexpr__ Fraction<> s<3, 19>[19] = {" + ", ".join(svals) + "};")
    out.append("template <>")
    out.append(f"__constexpr__ int shearIndexes<3, 19> = {len(SHEAR)};")
    out.append("template <>")
    out.append("__constexpr__ int shearViscIndexes<3, 19>[shearIndexes<3, 19>] = {"
               + ", ".join(str(s) for s in SHEAR) + "};")
    out.append("}  // namespace mrtdata")
    print("\n".join(out))


if __name__ == "__main__":
    main()
