// Thin C entry point around the reference's own run-summary logic (complab_diag::Diagnostics,
// complab3d_diagnostics.hh, which needs no Palabos), compiled from the reference sources where
// they lie (see Makefile target `ref`). TEST INFRASTRUCTURE ONLY: used to pin the host-side
// summary CSV, messages and final report to the reference's.
#include "complab3d_diagnostics.hh"

#include <cstring>
#include <string>

/* Records n_rows rows of n_fields fields (stats[row][field] = total, mean, min, max, held) with
 * the given conservation checks, writing the CSV to csv; the messages of every record() and the
 * final report go, NUL-terminated, into msgs and report. */
extern "C" void ref_diag_run(const char* csv, double tol, int n_checks, const char* const* exprs, int n_rows,
                             int n_fields, const char* const* names, const long* iters, const double* porosity,
                             const long* open_voxels, const double* stats, char* msgs, int msgs_len, char* report,
                             int report_len) {
    complab_diag::Diagnostics d;
    d.configure(true, csv, tol, true);
    for (int c = 0; c < n_checks; ++c) d.addConserve(exprs[c]);
    std::string all;
    for (int r = 0; r < n_rows; ++r) {
        complab_diag::Row row;
        row.iteration = iters[r];
        row.porosity = porosity[r];
        row.openVoxels = open_voxels[r];
        for (int f = 0; f < n_fields; ++f) {
            complab_diag::FieldStat st;
            const double* v = stats + ((size_t)r * n_fields + f) * 5;
            st.name = names[f];
            st.total = v[0]; st.mean = v[1]; st.minv = v[2]; st.maxv = v[3]; st.held = v[4];
            row.fields.push_back(st);
        }
        all += d.record(row);
    }
    const std::string rep = d.finalReport();
    std::strncpy(msgs, all.c_str(), (size_t)msgs_len - 1);
    msgs[msgs_len - 1] = 0;
    std::strncpy(report, rep.c_str(), (size_t)report_len - 1);
    report[report_len - 1] = 0;
}
