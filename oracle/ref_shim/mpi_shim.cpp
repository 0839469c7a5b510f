// Single-rank implementation of the MPI calls declared in mpi.h (oracle build only).
#include "mpi.h"
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <fcntl.h>
#include <unistd.h>

namespace {
std::vector<int>& type_sizes() {
    static std::vector<int> t = {0, 1, 1, (int)sizeof(int), (int)sizeof(unsigned), 4, 8, 4, 8, 8};
    return t;
}
int size_of(MPI_Datatype t) {
    if (t < 0 || t >= (int)type_sizes().size()) {
        std::fprintf(stderr, "mpi shim: unknown datatype %d\n", t);
        std::abort();
    }
    return type_sizes()[t];
}
[[noreturn]] void no_peer(const char* what) {
    std::fprintf(stderr, "mpi shim: %s called on a single-rank communicator\n", what);
    std::abort();
}
}  // namespace

int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) { std::fflush(stdout); std::exit(code == 0 ? 1 : code); }
int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm) {
    if (send != recv) std::memcpy(recv, send, (size_t)count * size_of(type));
    return MPI_SUCCESS;
}
int MPI_Alltoall(const void* send, int scount, MPI_Datatype stype, void* recv, int, MPI_Datatype, MPI_Comm) {
    if (send != recv) std::memcpy(recv, send, (size_t)scount * size_of(stype));
    return MPI_SUCCESS;
}
int MPI_Allgather(const void* send, int scount, MPI_Datatype stype, void* recv, int, MPI_Datatype, MPI_Comm) {
    if (send != recv) std::memcpy(recv, send, (size_t)scount * size_of(stype));
    return MPI_SUCCESS;
}
int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { no_peer("MPI_Send"); }
int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { no_peer("MPI_Recv"); }
int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { no_peer("MPI_Isend"); }
int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { no_peer("MPI_Irecv"); }
int MPI_Waitall(int n, MPI_Request*, MPI_Status*) {
    if (n != 0) no_peer("MPI_Waitall");
    return MPI_SUCCESS;
}
int MPI_Type_size(MPI_Datatype type, int* size) { *size = size_of(type); return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype* type) { *type = 0; return MPI_SUCCESS; }
int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
int MPI_Type_match_size(int, int size, MPI_Datatype* type) {
    type_sizes().push_back(size);
    *type = (int)type_sizes().size() - 1;
    return MPI_SUCCESS;
}
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype* out) {
    type_sizes().push_back(count * size_of(old));
    *out = (int)type_sizes().size() - 1;
    return MPI_SUCCESS;
}
int MPI_Type_create_struct(int count, const int* blocklens, const MPI_Aint* disps,
                           const MPI_Datatype* types, MPI_Datatype* out) {
    long long extent = 0;
    for (int i = 0; i < count; ++i) {
        long long end = disps[i] + (long long)blocklens[i] * size_of(types[i]);
        if (end > extent) extent = end;
    }
    type_sizes().push_back((int)extent);
    *out = (int)type_sizes().size() - 1;
    return MPI_SUCCESS;
}
int MPI_File_open(MPI_Comm, const char* name, int mode, MPI_Info, MPI_File* fh) {
    int flags = (mode & MPI_MODE_WRONLY) ? O_WRONLY : O_RDONLY;
    if (mode & MPI_MODE_CREATE) flags |= O_CREAT;
    int fd = ::open(name, flags, 0644);
    if (fd < 0) return 1;
    *fh = fd;
    return MPI_SUCCESS;
}
int MPI_File_close(MPI_File* fh) { ::close(*fh); *fh = -1; return MPI_SUCCESS; }
int MPI_File_write_at_all(MPI_File fh, MPI_Offset off, const void* buf, int count, MPI_Datatype type,
                          MPI_Status*) {
    size_t n = (size_t)count * size_of(type);
    return ::pwrite(fh, buf, n, off) == (ssize_t)n ? MPI_SUCCESS : 1;
}
int MPI_File_read_at_all(MPI_File fh, MPI_Offset off, void* buf, int count, MPI_Datatype type,
                         MPI_Status*) {
    size_t n = (size_t)count * size_of(type);
    return ::pread(fh, buf, n, off) == (ssize_t)n ? MPI_SUCCESS : 1;
}
