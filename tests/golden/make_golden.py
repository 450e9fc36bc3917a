"""Builds the golden fixtures under tests/golden/ from the reference's own data files.

Run once in a container that holds the reference checkout (read-only):

    python tests/golden/make_golden.py /path/to/pmsim

Nothing at test time reads the reference; the tests load the .npz/.json written here.
Sources (paths inside the pmsim project):
  * data/spo/test_von_mises_single_element_2d_ref.json   (HYPLAS, Qua4 1 IP, 5 steps)
  * data/spo/test_von_mises_2x2_elements_2d_ref.json     (HYPLAS, Qua8 4 IP, 5 steps)
  * data/spo/spo_754_footing_ref.json + spo_754_footing.msh (HYPLAS, Qua8 4 IP, 14 steps)
  * data/spo/spo_755_tensile_perf_plast_ref.json + spo_755_tensile.msh (Qua8 4 IP, 15 steps)
  * data/spo/spo_753_circ_plate_ref.json + spo_753_circ_plate.msh (axisymmetric Qua8 4 IP, 12 steps)
  * data/spo/spo_752_pres_sphere_collapse_ref.json (axisymmetric sphere on the SPO 7.5.1 mesh, 4 steps)
  * data/results/artificial/*.json, *.msh  (pmsim's own FemState output, uniform fields; the
    raw files are kept as femstate_*.json for the byte-level checkpoint test)
  * data/sgm/sgm_5d17_ref.json and tests/test_solid_smith_5d17_qua4_axisym.rs (axisymmetric Qua4)
  * tests/test_solid_smith_5d7_tri15_plane_strain.rs and smith_example_5d7_tri15 (Tri15, 12 IP)
  * tests/test_solid_bhatti_1d6_plane_stress.rs and the bhatti_example_1d6_bracket mesh (plane stress)
  * tests/test_solid_smith_5d11_qua4_plane_strain_uy.rs (inline expected displacements) and
    src/base/sample_meshes.rs (smith_example_5d11_qua4, smith_example_5d24_hex20 meshes)
  * data/meshes/test_solid_felippa_thick_cylinder_axisym.msh, test_durand_farias_example4_qua4.msh
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_msh(path):
    lines = [ln for ln in open(path).read().split("\n") if ln.strip() and not ln.lstrip().startswith("#")]
    ndim, npoint, ncell = map(int, lines[0].split())
    coords = np.array([[float(v) for v in ln.split()[2:2 + ndim]] for ln in lines[1:1 + npoint]])
    rows = [ln.split() for ln in lines[1 + npoint:1 + npoint + ncell]]
    kinds = sorted({r[2] for r in rows})
    cells = np.array([[int(v) for v in r[3:]] for r in rows], dtype=np.int64)
    return ndim, coords, cells, kinds[0]


def spo(ref, name, out, mesh=None):
    d = json.load(open(os.path.join(ref, "data/spo", name)))["all"]
    disp = np.array([s["displacement"] for s in d])  # (nstep, npoint, ndim)
    stress = np.array([s["stresses"] for s in d])  # (nstep, ncell, ngauss, ncomp) Voigt shear
    iters = np.array([len(s["iterations"]) for s in d])
    load = np.array([s["load_factor"] for s in d])
    arrs = dict(displacement=disp, stresses=stress, hyplas_iterations=iters, load_factor=load)
    if mesh is not None:
        ndim, coords, cells, kind = read_msh(os.path.join(ref, mesh))
        arrs.update(coords=coords, cells=cells, kind=np.array(kind))
    np.savez_compressed(os.path.join(HERE, out), **arrs)
    print("wrote", out, disp.shape, stress.shape)


def artificial(ref, stem, out):
    base = os.path.join(ref, "data/results/artificial")
    ndim, coords, cells, kind = read_msh(os.path.join(base, f"{stem}-mesh.msh"))
    us, sig, eps = [], [], []
    for i in range(3):
        st = json.load(open(os.path.join(base, f"{stem}-{i:020d}.json")))
        us.append(st["u"]["data"])
        sig.append([[ip["stress"]["vec"]["data"] for ip in c["solid"]] for c in st["gauss"]])
        eps.append([[ip["strain"]["vec"]["data"] for ip in c["solid"]] for c in st["gauss"]])
    np.savez_compressed(os.path.join(HERE, out), coords=coords, cells=cells, kind=np.array(kind),
                        u=np.array(us), stress=np.array(sig), strain=np.array(eps))
    print("wrote", out, np.array(sig).shape)


def rust_mesh(ref, fn_name):
    src = open(os.path.join(ref, "src/base/sample_meshes.rs")).read()
    i = src.index(f"pub fn {fn_name}()")
    j = src.index("\n    }\n", i)
    body = src[i:j]
    pts = re.findall(r"Point\s*\{\s*id:\s*(\d+),\s*marker:\s*-?\d+,\s*coords:\s*vec!\[([^\]]*)\]", body)
    cells = re.findall(r"Cell\s*\{[^}]*kind:\s*GeoKind::(\w+),\s*points:\s*vec!\[([^\]]*)\]", body)
    coords = np.array([[float(v) for v in c.split(",") if v.strip()] for _, c in pts])
    conn = np.array([[int(v) for v in c.split(",") if v.strip()] for _, c in cells], dtype=np.int64)
    return coords, conn, cells[0][0].lower()


def rust_array(path, var):
    src = open(path).read()
    i = src.index(f"let {var}")
    j = src.index("];", i)
    nums = re.findall(r"[-+]?\d+\.\d+(?:e[-+]?\d+)?", src[src.index("[", i):j])
    return np.array([float(v) for v in nums])


def main(ref):
    spo(ref, "test_von_mises_single_element_2d_ref.json", "spo_single_element_2d.npz")
    spo(ref, "test_von_mises_2x2_elements_2d_ref.json", "spo_2x2_elements_2d.npz",
        mesh="data/results/artificial/artificial-elastic-2d-qua8-mesh.msh")
    spo(ref, "spo_754_footing_ref.json", "spo_754_footing.npz", mesh="data/spo/spo_754_footing.msh")
    spo(ref, "spo_755_tensile_perf_plast_ref.json", "spo_755_tensile.npz", mesh="data/spo/spo_755_tensile.msh")
    artificial(ref, "artificial-elastic-2d-qua8", "artificial_2d_qua8.npz")
    artificial(ref, "artificial-elastic-2d", "artificial_2d_tri3.npz")
    artificial(ref, "artificial-elastic-3d", "artificial_3d_hex8.npz")
    # raw FemState files written by pmsim itself (byte-level checkpoint compatibility)
    import shutil
    for stem in ("artificial-elastic-2d-qua8", "artificial-elastic-3d"):
        for i in range(3):
            src = os.path.join(ref, "data/results/artificial", f"{stem}-{i:020d}.json")
            shutil.copyfile(src, os.path.join(HERE, f"femstate_{stem}_{i}.json"))
    print("copied FemState json files")
    coords, conn, kind = rust_mesh(ref, "smith_example_5d11_qua4")
    uu = rust_array(os.path.join(ref, "tests/test_solid_smith_5d11_qua4_plane_strain_uy.rs"), "uu_correct")
    np.savez_compressed(os.path.join(HERE, "smith_5d11_qua4.npz"), coords=coords, cells=conn, kind=np.array(kind),
                        uu_correct=uu)
    print("wrote smith_5d11_qua4.npz", coords.shape, conn.shape, uu.shape)
    coords, conn, kind = rust_mesh(ref, "smith_example_5d24_hex20")
    np.savez_compressed(os.path.join(HERE, "smith_5d24_hex20_mesh.npz"), coords=coords, cells=conn,
                        kind=np.array(kind))
    print("wrote smith_5d24_hex20_mesh.npz", coords.shape, conn.shape)
    # linear-elastic SGM runs with natural boundary conditions: mesh, cell attributes, expected U
    for fn, test, out in [("smith_example_5d2_tri3", "test_solid_smith_5d2_tri3_plane_strain.rs", "smith_5d2_tri3"),
                          ("smith_example_5d7_tri15", "test_solid_smith_5d7_tri15_plane_strain.rs",
                           "smith_5d7_tri15"),
                          ("smith_example_5d15_qua8", "test_solid_smith_5d15_qua8_plane_strain.rs",
                           "smith_5d15_qua8"),
                          ("smith_example_5d30_tet4", "test_solid_smith_5d30_tet4_3d.rs", "smith_5d30_tet4"),
                          ("smith_example_5d24_hex20", "test_solid_smith_5d24_hex20_3d.rs", "smith_5d24_hex20"),
                          ("smith_example_5d27_qua9", "test_solid_smith_5d27_qua9_plane_strain.rs",
                           "smith_5d27_qua9")]:
        coords, conn, kind = rust_mesh(ref, fn)
        src = open(os.path.join(ref, "src/base/sample_meshes.rs")).read()
        i = src.index(f"pub fn {fn}()")
        body = src[i:src.index("\n    }\n", i)]
        attr = np.array([int(a) for a in re.findall(r"Cell\s*\{\s*id:\s*\d+,\s*attribute:\s*(\d+)", body)])
        uu = rust_array(os.path.join(ref, "tests", test), "uu_correct")
        np.savez_compressed(os.path.join(HERE, out + ".npz"), coords=coords, cells=conn, kind=np.array(kind),
                            attribute=attr, uu_correct=uu)
        print("wrote", out, coords.shape, conn.shape, uu.shape)
    # SGM 5.17 axisymmetric Qua4 (9 IP, two layers, point loads): mesh, cell attributes, expected U of
    # the test, and Smith-Griffiths' own element stiffness matrices, displacements and IP stresses
    coords, conn, kind = rust_mesh(ref, "smith_example_5d17_qua4")
    src = open(os.path.join(ref, "src/base/sample_meshes.rs")).read()
    i = src.index("pub fn smith_example_5d17_qua4()")
    body = src[i:src.index("\n    }\n", i)]
    attr = np.array([int(a) for a in re.findall(r"Cell\s*\{\s*id:\s*\d+,\s*attribute:\s*(\d+)", body)])
    uu = rust_array(os.path.join(ref, "tests", "test_solid_smith_5d17_qua4_axisym.rs"), "uu_correct")
    sgm = json.load(open(os.path.join(ref, "data/sgm/sgm_5d17_ref.json")))["all"][0]
    np.savez_compressed(os.path.join(HERE, "smith_5d17_qua4_axisym.npz"), coords=coords, cells=conn,
                        kind=np.array(kind), attribute=attr, uu_correct=uu,
                        sgm_stiffness=np.array(sgm["stiffness"]), sgm_displacement=np.array(sgm["displacement"]),
                        sgm_stresses=np.array(sgm["stresses"]))
    print("wrote smith_5d17_qua4_axisym", coords.shape, conn.shape, uu.shape)
    # Bhatti 1.6 bracket in plane stress (Tri3, thickness 0.25, linear elastic)
    coords, conn, kind = rust_mesh(ref, "bhatti_example_1d6_bracket")
    uu = rust_array(os.path.join(ref, "tests", "test_solid_bhatti_1d6_plane_stress.rs"), "uu_correct")
    np.savez_compressed(os.path.join(HERE, "bhatti_1d6_plane_stress.npz"), coords=coords, cells=conn,
                        kind=np.array(kind), uu_correct=uu)
    print("wrote bhatti_1d6_plane_stress", coords.shape, conn.shape, uu.shape)
    # SPO 7.5.1 pressurised cylinder (reduced-system method, internal pressure, von Mises)
    spo(ref, "spo_751_pres_cylin_ref.json", "spo_751_pres_cylin.npz", mesh="data/spo/spo_751_pres_cylin_qua4.msh")
    spo(ref, "spo_753_circ_plate_ref.json", "spo_753_circ_plate.npz", mesh="data/spo/spo_753_circ_plate.msh")
    spo(ref, "spo_752_pres_sphere_collapse_ref.json", "spo_752_pres_sphere_collapse.npz")
    # meshes of the linear-elastic benchmark tests that read them from data/meshes
    for stem, out in [("test_solid_felippa_thick_cylinder_axisym", "felippa_thick_cylinder_axisym"),
                      ("test_durand_farias_example4_qua4", "durand_farias_example4_qua4")]:
        ndim, coords, cells, kind = read_msh(os.path.join(ref, "data/meshes", stem + ".msh"))
        np.savez_compressed(os.path.join(HERE, out + ".npz"), coords=coords, cells=cells, kind=np.array(kind))
        print("wrote", out, coords.shape, cells.shape, kind)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the pmsim source tree>")
    main(sys.argv[1])
