// Thin C entry point around the reference's own equilibrium solver (EquilibriumChemistry:
// positive-continued-fraction fixed point with Anderson acceleration), compiled from the
// reference sources where they lie with the reference's own single-cell Palabos stub
// (see Makefile target `ref`). TEST INFRASTRUCTURE ONLY: used to pin the speciation restatement
// and the GPU Newton-Raphson kernel to the reference's root.
#include "palabos_stub.hh"
using namespace plb;
#include "complab3d_processors_part4_eqsolver.hh"

#include <string>
#include <vector>

// stoich: [ns][nc] row-major; comp_species[j] = species index of component j or -1.
extern "C" int ref_eq_solve(int ns, int nc, const double* stoich, const double* logK, const int* comp_species,
                            double tol, int max_iter, const double* conc_in, double* conc_out, int* converged,
                            int* iterations) {
    EquilibriumChemistry<double> eq;
    std::vector<std::string> sn(ns), cn(nc);
    for (int i = 0; i < ns; ++i) sn[i] = "s" + std::to_string(i);
    for (int j = 0; j < nc; ++j) cn[j] = comp_species[j] >= 0 ? sn[comp_species[j]] : "c" + std::to_string(j);
    eq.setSpeciesNames(sn);
    eq.setComponentNames(cn);
    std::vector<double> lk(logK, logK + ns);
    eq.setLogK(lk);
    std::vector<std::vector<double>> S(ns, std::vector<double>(nc));
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j < nc; ++j) S[i][j] = stoich[i * nc + j];
    eq.setStoichiometryMatrix(S);
    eq.setTolerance(tol);
    eq.setMaxIterations(max_iter);
    std::vector<double> c(conc_in, conc_in + ns);
    std::vector<double> r = eq.calculate_species_concentrations(c);
    for (int i = 0; i < ns; ++i) conc_out[i] = r[i];
    *converged = eq.didConverge() ? 1 : 0;
    *iterations = (int)eq.getLastIterations();
    return 0;
}
