"""Run directories for the CompLaB.xml cases of tests/golden/cases: the XML copied beside an
input/ folder holding its geometry file, written from a seeded map in the reference's .dat order
(interior x-planes, x slowest, z fastest, one integer per line)."""
import os
import shutil

import numpy as np

HERE = os.path.join(os.path.dirname(__file__), "golden", "cases")


def write_dat(path, inner):
    with open(path, "w") as f:
        f.write("\n".join(str(int(v)) for v in np.asarray(inner).ravel()))
        f.write("\n")


def carbonate_duct_map():
    nx, ny, nz = 20, 12, 10
    m = np.full((nx, ny, nz), 2, np.int8)
    m[:, 0, :] = m[:, -1, :] = 1
    m[:, :, 0] = m[:, :, -1] = 1
    m[6:9, 4:8, 3:6] = 1
    m[13:15, 2:5, 5:9] = 0
    return m


def biofilm_flow_map(clb):
    nx, ny, nz = 22, 12, 11
    m = clb.sphere_pack(nx, ny, nz, 0.55, 2.0, 3.0, 33, "yz").reshape(nx, ny, nz)
    rng = np.random.default_rng(33)
    pore = np.argwhere(m == 2)
    pore = pore[(pore[:, 0] > 2) & (pore[:, 0] < nx - 3)]
    pick = pore[rng.choice(len(pore), size=40, replace=False)]
    for k, (x, y, z) in enumerate(pick):
        m[x, y, z] = 3 if k % 2 == 0 else 4
    return m


def graphnet_duct_map():
    nx, ny, nz = 18, 10, 9
    m = np.full((nx, ny, nz), 2, np.int8)
    m[:, 0, :] = m[:, -1, :] = 1
    m[:, :, 0] = m[:, :, -1] = 1
    m[5:7, 3:6, 2:5] = 1
    m[11:13, 5:8, 4:7] = 0
    m[8:11, 2:5, 3:7] = 3  # the biofilm patch
    return m


def run_dir(tmp, name, inner):
    d = os.path.join(str(tmp), name)
    os.makedirs(os.path.join(d, "input"), exist_ok=True)
    shutil.copy(os.path.join(HERE, name + ".xml"), os.path.join(d, "CompLaB.xml"))
    fname = {"carbonate_duct": "duct.dat", "biofilm_flow": "pack.dat", "graphnet_duct": "duct.dat"}[name]
    write_dat(os.path.join(d, "input", fname), inner)
    if name == "graphnet_duct":
        shutil.copy(os.path.join(os.path.dirname(HERE), "srg", "uptake_growth.srg"), os.path.join(d, "input", "organism.srg"))
        gnn = os.path.join(os.path.dirname(HERE), "gnn")
        shutil.copy(os.path.join(gnn, "extent_growth.gnn"), os.path.join(d, "input", "organism.gnn"))
        shutil.copy(os.path.join(gnn, "abiotic_extent.gnn"), os.path.join(d, "input", "abiotic.gnn"))
    return os.path.join(d, "CompLaB.xml")


def surrogate_case(tmp, inner):
    """The graph-network duct with its organism turned into a surrogate organism: reaction_type
    surrogate, a <surrogate> block naming input/organism.srg, the uptake parameters in the microbe
    block; the abiotic network stays."""
    xml = run_dir(tmp, "graphnet_duct", inner)
    text = open(xml).read()
    text = text.replace("<network_file>input/organism.gnn</network_file>", "")
    text = text.replace("<graphnet>", "<surrogate>\n        <enabled>true</enabled>\n"
                        "        <weights_file>input/organism.srg</weights_file>\n    </surrogate>\n    <graphnet>")
    text = text.replace("<reaction_type>graphnet</reaction_type>",
                        "<reaction_type>surrogate</reaction_type>\n"
                        "            <half_saturation_constants>0.05 0.1 0.02 0.2</half_saturation_constants>\n"
                        "            <fba_maximum_uptake_flux>10 5 0 0</fba_maximum_uptake_flux>\n"
                        "            <biomass_molar_mass>24.6</biomass_molar_mass>\n"
                        "            <decay_coefficient>2e-6</decay_coefficient>")
    text = text.replace("<initial_densities>60</initial_densities>", "<initial_densities>0.03</initial_densities>")
    out = os.path.join(os.path.dirname(xml), "surrogate.xml")
    open(out, "w").write(text)
    return out
