// mdi.cpp -- the command set of libERI's MDI plugin, without the transport.
//
// The reference plugin (src/interface/liberi_mdi_api.F90) registers the
// commands of initialize_mdi (:194-224) and answers them in execute_command
// (:272-428): basis, geometry and Schwarz data arrive with '>' commands and
// are accumulated in a persistent state, '>SCHWZ_INT' sets up the handle
// (liberi_setup), '>AO_DENS' delivers D, '<FOCK' builds this rank's partial F,
// reduces it over the ranks (MPI_Reduce) and sends it.  Here the state
// machine is a C-ABI object: a transport shim (an MDI plugin entry point
// linked against the MDI library) asks liberi_c_mdi_payload how many elements
// of which type a command carries, receives or sends them with MDI, and calls
// liberi_c_mdi_execute; the sum of the ranks' partial F is the shim's (MPI or
// NCCL), as the reference's caller-side reduction.
#include <cstring>
#include <new>
#include <algorithm>
#include <string>
#include <vector>

#include "../../include/liberi_b200.h"
#include "engine.h"

namespace liberi {
int set_error(int code, const char *msg);
}

using liberi::set_error;

struct liberi_mdi_s {
    liberi_handle handle = nullptr;
    int32_t rank = 0, nprocs = 1;
    int32_t natoms = 0, num_bas = 0, nsh = 0, mxgtot = 0;
    std::string typscf;
    std::vector<int32_t> ang_mom, contr_num, sh_loc, atom_num, atom_loc, start_bas, end_bas;
    std::vector<double> exponents, coef_s, coef_p, coef_d, coef_f, coords, schwrz;
    std::vector<double> density, density_b;
    std::vector<double> fock_b;  // beta partial F of the last open-shell '<FOCK'
    liberi_comm comm = nullptr;  // NCCL sum of the ranks' partials, or none (the shim sums)
};

namespace {

enum Kind { K_EXIT, K_EXIT_CONVERGED, K_TYPSCF, K_SCALAR, K_SHELL_INT, K_PRIM_DOUBLE, K_COORDS, K_SCHWZ,
            K_DENS, K_DENS_B, K_FOCK, K_FOCK_B, K_UNKNOWN };

struct Cmd {
    Kind kind;
    int32_t *scalar;
    std::vector<int32_t> *ivec;
    std::vector<double> *dvec;
};

// trailing blanks are not part of a command (the reference trims them)
std::string trimmed(const char *c) {
    std::string s(c ? c : "");
    while (!s.empty() && (s.back() == ' ' || s.back() == '\0')) s.pop_back();
    return s;
}

Cmd classify(liberi_mdi_s *s, const std::string &c) {
    if (c == "EXIT") return {K_EXIT, nullptr, nullptr, nullptr};
    if (c == "EXIT_CONVERGED") return {K_EXIT_CONVERGED, nullptr, nullptr, nullptr};
    if (c == ">TYPSCF") return {K_TYPSCF, nullptr, nullptr, nullptr};
    if (c == ">NATOMS") return {K_SCALAR, &s->natoms, nullptr, nullptr};
    if (c == ">NUM_BAS") return {K_SCALAR, &s->num_bas, nullptr, nullptr};
    if (c == ">NSH") return {K_SCALAR, &s->nsh, nullptr, nullptr};
    if (c == ">mxgtot") return {K_SCALAR, &s->mxgtot, nullptr, nullptr};
    if (c == ">RANK_ID") return {K_SCALAR, &s->rank, nullptr, nullptr};
    if (c == ">NUM_PROCS") return {K_SCALAR, &s->nprocs, nullptr, nullptr};
    if (c == ">ANGM") return {K_SHELL_INT, nullptr, &s->ang_mom, nullptr};
    if (c == ">CONTR") return {K_SHELL_INT, nullptr, &s->contr_num, nullptr};
    if (c == ">SHLLOC") return {K_SHELL_INT, nullptr, &s->sh_loc, nullptr};
    if (c == ">ATMNUM") return {K_SHELL_INT, nullptr, &s->atom_num, nullptr};
    if (c == ">ATMLOC") return {K_SHELL_INT, nullptr, &s->atom_loc, nullptr};
    if (c == ">SBAS") return {K_SHELL_INT, nullptr, &s->start_bas, nullptr};
    if (c == ">EBAS") return {K_SHELL_INT, nullptr, &s->end_bas, nullptr};
    if (c == ">EXPON") return {K_PRIM_DOUBLE, nullptr, nullptr, &s->exponents};
    if (c == ">CONTR_COEF_S") return {K_PRIM_DOUBLE, nullptr, nullptr, &s->coef_s};
    if (c == ">CONTR_COEF_P") return {K_PRIM_DOUBLE, nullptr, nullptr, &s->coef_p};
    if (c == ">CONTR_COEF_D") return {K_PRIM_DOUBLE, nullptr, nullptr, &s->coef_d};
    if (c == ">CONTR_COEF_F") return {K_PRIM_DOUBLE, nullptr, nullptr, &s->coef_f};
    if (c == ">COORDS") return {K_COORDS, nullptr, nullptr, &s->coords};
    if (c == ">SCHWZ_INT") return {K_SCHWZ, nullptr, nullptr, &s->schwrz};
    if (c == ">AO_DENS") return {K_DENS, nullptr, nullptr, &s->density};
    if (c == ">AO_DENS_B") return {K_DENS_B, nullptr, nullptr, &s->density_b};
    if (c == "<FOCK") return {K_FOCK, nullptr, nullptr, nullptr};
    if (c == "<FOCK_B") return {K_FOCK_B, nullptr, nullptr, nullptr};
    return {K_UNKNOWN, nullptr, nullptr, nullptr};
}

int64_t ntri(const liberi_mdi_s *s) { return (int64_t)s->num_bas * (s->num_bas + 1) / 2; }

void payload_of(const liberi_mdi_s *s, Kind k, int32_t *type, int64_t *count) {
    *type = LIBERI_MDI_NONE;
    *count = 0;
    switch (k) {
        case K_TYPSCF: *type = LIBERI_MDI_CHAR; *count = 10; break;
        case K_SCALAR: *type = LIBERI_MDI_INT; *count = 1; break;
        case K_SHELL_INT: *type = LIBERI_MDI_INT; *count = s->nsh; break;
        case K_PRIM_DOUBLE: *type = LIBERI_MDI_DOUBLE; *count = (int64_t)s->mxgtot * s->nsh; break;
        case K_COORDS: *type = LIBERI_MDI_DOUBLE; *count = 3 * (int64_t)s->natoms; break;
        case K_SCHWZ: *type = LIBERI_MDI_DOUBLE; *count = (int64_t)s->nsh * (s->nsh + 1) / 2; break;
        case K_DENS: case K_DENS_B: case K_FOCK: case K_FOCK_B: *type = LIBERI_MDI_DOUBLE; *count = ntri(s); break;
        default: break;
    }
}

const double *or_null(const std::vector<double> &v) { return v.empty() ? nullptr : v.data(); }
const int32_t *or_null(const std::vector<int32_t> &v) { return v.empty() ? nullptr : v.data(); }

}  // namespace

extern "C" {

int liberi_c_mdi_create(liberi_mdi *state, int32_t my_rank, int32_t num_procs) {
    if (!state || num_procs < 1 || my_rank < 0 || my_rank >= num_procs)
        return set_error(LIBERI_E_ARG, "liberi_mdi_create: bad arguments");
    liberi_mdi s = new (std::nothrow) liberi_mdi_s();
    if (!s) return set_error(LIBERI_E_NOMEM, "liberi_mdi_create: out of host memory");
    s->rank = my_rank;
    s->nprocs = num_procs;
    *state = s;
    return LIBERI_OK;
}

int liberi_c_mdi_payload(liberi_mdi s, const char *command, int32_t *type, int64_t *count) {
    if (!s || !command || !type || !count) return set_error(LIBERI_E_ARG, "liberi_mdi_payload: null argument");
    const Cmd c = classify(s, trimmed(command));
    if (c.kind == K_UNKNOWN) return set_error(LIBERI_E_ARG, "MDI command not recognized");
    payload_of(s, c.kind, type, count);
    return LIBERI_OK;
}

int liberi_c_mdi_execute(liberi_mdi s, const char *command, void *buffer, int64_t count, int32_t *terminate) {
    if (!s || !command) return set_error(LIBERI_E_ARG, "liberi_mdi_execute: null argument");
    if (terminate) *terminate = 0;
    const std::string name = trimmed(command);
    const Cmd c = classify(s, name);
    if (c.kind == K_UNKNOWN) return set_error(LIBERI_E_ARG, ("MDI command not recognized: " + name).c_str());
    int32_t type = 0;
    int64_t want = 0;
    payload_of(s, c.kind, &type, &want);
    if (want > 0 && (!buffer || count != want)) {
        const std::string m = "MDI command " + name + ": payload of " + std::to_string(count) + " elements, expected " +
                              std::to_string(want);
        return set_error(LIBERI_E_SIZE, m.c_str());
    }
    switch (c.kind) {
        case K_EXIT:
            if (terminate) *terminate = 1;
            return LIBERI_OK;
        case K_EXIT_CONVERGED:  // liberi_mdi_api.F90:286-290
            if (s->handle) {
                liberi_c_cleanup(s->handle);
                liberi_c_destroy(s->handle);
                s->handle = nullptr;
            }
            if (terminate) *terminate = 1;
            return LIBERI_OK;
        case K_TYPSCF: {
            s->typscf.assign((const char *)buffer, 10);
            return LIBERI_OK;
        }
        case K_SCALAR:
            *c.scalar = *(const int32_t *)buffer;
            if (s->nprocs < 1 || s->rank < 0 || s->rank >= s->nprocs)
                return set_error(LIBERI_E_ARG, "MDI: rank/num_procs out of range");
            return LIBERI_OK;
        case K_SHELL_INT:
            c.ivec->assign((const int32_t *)buffer, (const int32_t *)buffer + want);
            return LIBERI_OK;
        case K_PRIM_DOUBLE: case K_COORDS: case K_DENS: case K_DENS_B:
            c.dvec->assign((const double *)buffer, (const double *)buffer + want);
            return LIBERI_OK;
        case K_SCHWZ: {  // liberi_mdi_api.F90:355-389: set up, then drop the accumulated arrays
            c.dvec->assign((const double *)buffer, (const double *)buffer + want);
            if (!s->handle) {
                int rc = liberi_c_create(&s->handle);
                if (rc) return rc;
            }
            // with an NCCL communicator, each rank builds on its communicator's device
            if (s->comm) liberi_c_set_option(s->handle, "device", (double)liberi::comm_device(s->comm));
            int rc = liberi_c_setup(s->handle, s->nsh, s->natoms, s->num_bas, s->mxgtot, or_null(s->ang_mom),
                                    or_null(s->contr_num), or_null(s->sh_loc), or_null(s->atom_num),
                                    or_null(s->atom_loc), or_null(s->start_bas), or_null(s->end_bas),
                                    or_null(s->exponents), or_null(s->coef_s), or_null(s->coef_p), or_null(s->coef_d),
                                    or_null(s->coef_f), or_null(s->coords), or_null(s->schwrz), s->rank, s->nprocs);
            for (auto *v : {&s->ang_mom, &s->contr_num, &s->sh_loc, &s->atom_num, &s->atom_loc, &s->start_bas,
                            &s->end_bas})
                std::vector<int32_t>().swap(*v);
            for (auto *v : {&s->exponents, &s->coef_s, &s->coef_p, &s->coef_d, &s->coef_f, &s->coords, &s->schwrz})
                std::vector<double>().swap(*v);
            return rc;
        }
        case K_FOCK: {  // this rank's partial F (liberi_mdi_api.F90:405-420 before its MPI_Reduce)
            if (!s->handle) return set_error(LIBERI_E_STATE, "MDI <FOCK before >SCHWZ_INT set the handle up");
            if ((int64_t)s->density.size() != want)
                return set_error(LIBERI_E_STATE, "MDI <FOCK before >AO_DENS delivered the density");
            s->fock_b.clear();
            if ((int64_t)s->density_b.size() != want) {  // closed shell
                int rc = liberi_c_fock_build(s->handle, s->density.data(), (double *)buffer, (int32_t)want);
                if (!rc && s->comm) rc = liberi_c_comm_reduce_host(s->comm, (double *)buffer, (double *)buffer, want);
                return rc;
            }
            // open shell ('>AO_DENS_B' delivered the beta density): alpha F now,
            // beta F kept for '<FOCK_B' (the reference registers both commands,
            // liberi_mdi_api.F90:395-421, but builds closed-shell F only)
            s->fock_b.assign((size_t)want, 0.0);
            int rc = liberi_c_fock_build_uhf(s->handle, s->density.data(), s->density_b.data(), (double *)buffer,
                                             s->fock_b.data(), (int32_t)want);
            if (!rc && s->comm) rc = liberi_c_comm_reduce_host(s->comm, (double *)buffer, (double *)buffer, want);
            if (!rc && s->comm) rc = liberi_c_comm_reduce_host(s->comm, s->fock_b.data(), s->fock_b.data(), want);
            if (rc) s->fock_b.clear();
            return rc;
        }
        case K_FOCK_B:
            if ((int64_t)s->fock_b.size() != want)
                return set_error(LIBERI_E_STATE, "MDI <FOCK_B needs an open-shell <FOCK first (>AO_DENS_B, then <FOCK)");
            std::copy(s->fock_b.begin(), s->fock_b.end(), (double *)buffer);
            return LIBERI_OK;
        default:
            return set_error(LIBERI_E_ARG, "MDI command not recognized");
    }
}

int liberi_c_mdi_set_comm(liberi_mdi s, liberi_comm comm) {
    if (!s) return set_error(LIBERI_E_ARG, "liberi_mdi_set_comm: null state");
    s->comm = comm;
    return LIBERI_OK;
}

int liberi_c_mdi_destroy(liberi_mdi s) {
    if (!s) return set_error(LIBERI_E_ARG, "liberi_mdi_destroy: null state");
    if (s->handle) liberi_c_destroy(s->handle);
    delete s;
    return LIBERI_OK;
}

}  // extern "C"
