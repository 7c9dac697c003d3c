/* Minimal declarations of the MDI calls the plugin shim uses, written for a
 * compile check of gms_liberi_b200/mdi/liberi_mdi_plugin.c where the MDI
 * library is not installed (signatures as the shim calls them). */
#ifndef LIBERI_TEST_STUB_MDI_H
#define LIBERI_TEST_STUB_MDI_H
typedef int MDI_Comm;
typedef int MDI_Datatype;
#define MDI_INT 1
#define MDI_DOUBLE 2
#define MDI_CHAR 3
#define MDI_COMMAND_LENGTH 256
#define MDI_ENGINE 2
int MDI_Recv(void *buf, int count, MDI_Datatype type, MDI_Comm comm);
int MDI_Send(const void *buf, int count, MDI_Datatype type, MDI_Comm comm);
int MDI_Recv_command(char *command, MDI_Comm comm);
int MDI_Set_plugin_state(void *state);
int MDI_Get_role(int *role);
int MDI_Register_node(const char *node);
int MDI_Register_command(const char *node, const char *command);
int MDI_Accept_communicator(MDI_Comm *comm);
#endif
