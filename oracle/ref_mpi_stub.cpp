// Single-process stand-ins for the MPI routines the reference's Index.cpp and
// node.cpp reference.  The oracle only drives single-process code paths, so
// reaching any of these is a usage error: they print and return failure
// rather than pretend to communicate.  TEST INFRASTRUCTURE ONLY.
#include <cstdio>
#include "mpi.h"

static int refuse(const char* name) {
    std::fprintf(stderr, "oracle: MPI routine %s reached in a single-process build\n", name);
    return 1;
}
extern "C" {
int MPI_Abort(MPI_Comm, int) { return refuse("MPI_Abort"); }
int MPI_Barrier(MPI_Comm) { return refuse("MPI_Barrier"); }
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return refuse("MPI_Bcast"); }
int MPI_Comm_get_attr(MPI_Comm, int, void*, int* flag) {
    if (flag) *flag = 0;
    return 0;
}
int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { return refuse("MPI_Irecv"); }
int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { return refuse("MPI_Isend"); }
int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return refuse("MPI_Recv"); }
int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return refuse("MPI_Send"); }
int MPI_Test(MPI_Request*, int* flag, MPI_Status*) {
    if (flag) *flag = 1;
    return refuse("MPI_Test");
}
int MPI_Wait(MPI_Request*, MPI_Status*) { return refuse("MPI_Wait"); }
int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return refuse("MPI_Waitall"); }
}
