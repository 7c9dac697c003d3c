/* liberi_mdi_plugin.c -- MDI plugin entry points of the engine for GAMESS.
 *
 * Replaces the reference's src/interface/liberi_mdi_api.F90 (MDI_Plugin_init_ERI,
 * MDI_Plugin_open_ERI, MDI_Plugin_close_ERI): registers the same commands on
 * node @DEFAULT, then answers the driver.  The command state machine is the
 * library's liberi_c_mdi_* object; this file only moves payloads with MDI.
 * The ranks' partial Fock matrices are summed on the GPUs: rank 0 makes an
 * NCCL id (liberi_c_comm_unique_id), MPI_Bcast hands it to every rank, each
 * rank creates its communicator on its own device and attaches it to the
 * state (liberi_c_mdi_set_comm), so '<FOCK' / '<FOCK_B' come back summed and
 * rank 0 sends them (the reference sums with MPI_Reduce to rank 0,
 * liberi_mdi_api.F90:411-414; that path remains if NCCL cannot be set up).
 * Build it against the MDI library and an MPI C compiler, and link with
 * -lliberi_b200:
 *
 *     mpicc -shared -fPIC -I<mdi>/include -I<repo>/include liberi_mdi_plugin.c \
 *           -L<repo>/gms_liberi_b200/_build -lliberi_b200 -lmdi -o libliberi_mdi.so
 *
 * The state persists across plugin launches (GAMESS launches the plugin once
 * for setup and once per SCF iteration); 'EXIT_CONVERGED' releases the handle. */
#include <mdi.h>
#include <mpi.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "liberi_b200.h"

static liberi_mdi g_state = NULL;
static liberi_comm g_nccl = NULL; /* NCCL sum of the partial F, or NULL (MPI_Reduce) */
static MDI_Comm g_comm;
static MPI_Comm g_world;

static const char *k_commands[] = {
    "EXIT", "EXIT_CONVERGED", "<FOCK", ">FOCK", ">NATOMS", ">RANK_ID", ">NUM_PROCS", ">NUM_BAS", ">NSH",
    ">mxgtot", ">ANGM", "<COORDS", ">COORDS", ">CONTR", ">SHLLOC", ">ATMNUM", ">ATMLOC", ">SBAS", ">EBAS",
    ">EXPON", ">CONTR_COEF_S", ">CONTR_COEF_P", ">CONTR_COEF_D", ">CONTR_COEF_F", ">SCHWZ_INT", ">AO_DENS",
    ">TYPSCF", "<FOCK_B", ">FOCK_B", ">AO_DENS_B"};

static void report(const char *cmd, int rc) {
    char msg[512];
    liberi_c_last_error(msg, sizeof msg);
    fprintf(stderr, "libERI MDI: command %s failed (%d): %s\n", cmd, rc, msg);
}

static int mdi_type(int32_t t) { return t == LIBERI_MDI_INT ? MDI_INT : (t == LIBERI_MDI_DOUBLE ? MDI_DOUBLE : MDI_CHAR); }
static MPI_Datatype mpi_type(int32_t t) {
    return t == LIBERI_MDI_INT ? MPI_INT : (t == LIBERI_MDI_DOUBLE ? MPI_DOUBLE : MPI_CHAR);
}
static size_t elem_size(int32_t t) { return t == LIBERI_MDI_INT ? 4 : (t == LIBERI_MDI_DOUBLE ? 8 : 1); }

/* one command: receive ('>') and broadcast, or compute and reduce ('<') */
static int execute(const char *command, int *terminate) {
    int32_t type = 0, term = 0;
    int64_t count = 0;
    int rank = 0, ierr = 0, rc;
    MPI_Comm_rank(g_world, &rank);
    rc = liberi_c_mdi_payload(g_state, command, &type, &count);
    if (rc) {
        report(command, rc);
        return rc;
    }
    void *buf = count > 0 ? malloc((size_t)count * elem_size(type)) : NULL;
    if (command[0] == '>' && count > 0) {
        if (rank == 0) MDI_Recv(buf, (int)count, mdi_type(type), g_comm);
        MPI_Bcast(buf, (int)count, mpi_type(type), 0, g_world);
    }
    rc = liberi_c_mdi_execute(g_state, command, buf, count, &term);
    if (rc) report(command, rc);
    if (command[0] == '<' && count > 0 && rc == 0) {
        if (g_nccl) {  /* the library summed the partials over NCCL */
            if (rank == 0) MDI_Send(buf, (int)count, mdi_type(type), g_comm);
        } else {
            void *sum = rank == 0 ? malloc((size_t)count * elem_size(type)) : NULL;
            MPI_Reduce(buf, sum, (int)count, mpi_type(type), MPI_SUM, 0, g_world);
            if (rank == 0) {
                MDI_Send(sum, (int)count, mdi_type(type), g_comm);
                free(sum);
            }
        }
    }
    free(buf);
    *terminate = term;
    (void)ierr;
    return rc;
}

static int launch(void *plugin_state) {
    int rank = 0, size = 1, role = 0;
    MDI_Set_plugin_state(plugin_state);
    MDI_MPI_get_world_comm(&g_world);
    MPI_Comm_rank(g_world, &rank);
    MPI_Comm_size(g_world, &size);
    if (!g_state) {
        if (liberi_c_mdi_create(&g_state, rank, size) != LIBERI_OK) return 1;
        /* NCCL communicator over the ranks' devices (one rank per device) */
        uint8_t id[LIBERI_COMM_ID_BYTES];
        int ok = rank == 0 ? liberi_c_comm_unique_id(id) == LIBERI_OK : 1, all = 0;
        MPI_Bcast(&ok, 1, MPI_INT, 0, g_world);
        if (ok) {
            MPI_Bcast(id, LIBERI_COMM_ID_BYTES, MPI_BYTE, 0, g_world);
            ok = liberi_c_comm_create(&g_nccl, id, rank, size, -1) == LIBERI_OK;
        }
        MPI_Allreduce(&ok, &all, 1, MPI_INT, MPI_MIN, g_world);
        if (all && g_nccl) {
            liberi_c_mdi_set_comm(g_state, g_nccl);
        } else {  /* some rank could not join: sum with MPI as the reference does */
            if (g_nccl) liberi_c_comm_destroy(g_nccl);
            g_nccl = NULL;
        }
    }
    MDI_Get_role(&role);
    if (role != MDI_ENGINE) fprintf(stderr, "libERI MDI: must run as an ENGINE\n");
    MDI_Register_node("@DEFAULT");
    for (size_t i = 0; i < sizeof k_commands / sizeof k_commands[0]; i++)
        MDI_Register_command("@DEFAULT", k_commands[i]);
    MDI_Accept_communicator(&g_comm);
    char command[MDI_COMMAND_LENGTH + 1];
    for (;;) {
        int terminate = 0;
        if (rank == 0) MDI_Recv_command(command, g_comm);
        MPI_Bcast(command, MDI_COMMAND_LENGTH, MPI_CHAR, 0, g_world);
        command[MDI_COMMAND_LENGTH] = '\0';
        execute(command, &terminate);
        if (terminate) break;
    }
    return 0;
}

int MDI_Plugin_init_ERI(void *plugin_state) { return launch(plugin_state); }
int MDI_Plugin_open_ERI(void *plugin_state) { return launch(plugin_state); }
int MDI_Plugin_close_ERI(void) { return 0; }
