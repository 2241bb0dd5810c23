// Definitions the reference's CPU sources expect from their Fortran host
// (FHI-aims): the mpi_tasks module variables named in pass_mod_var.h.  Linked
// into oracle/_ref/ only, so that the reference compiles as a standalone
// library.  Test infrastructure.
extern "C++" {
int __mpi_tasks_MOD_n_tasks = 1;
int __mpi_tasks_MOD_myid = 0;
}
