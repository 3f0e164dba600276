/*
 * Single-rank stand-in for the MPI interface, written for this project.
 *
 * TEST INFRASTRUCTURE ONLY: it lets the reference GLAC sources compile and run
 * as one process so that they can serve as the parity oracle and the CPU
 * baseline.  With one rank every neighbour is the process itself, so
 *   - point-to-point calls (Sendrecv, Isend/Irecv/Wait) are self-copies,
 *   - reductions (Allreduce, Reduce) copy the send buffer to the receive buffer,
 *   - MPI-IO (File_open/read_at/write_at/close) maps onto pread/pwrite.
 * Only the subset of MPI used by GLAC's sources is provided.
 */
#ifndef GLAC_ORACLE_MPISHIM_H
#define GLAC_ORACLE_MPISHIM_H

#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <fcntl.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Group;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef int MPI_File;
struct MPI_Status { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; };
typedef int MPI_Request;

#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_DOUBLE 8
#define MPI_BYTE 1
#define MPI_SUM 1
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_SUCCESS 0

namespace glac_mpishim {
/* One outstanding non-blocking send / receive pair is enough: GLAC always posts
 * exactly one Isend and one Irecv before waiting on both. */
struct Pending { const void *send; void *recv; size_t bytes_send; size_t bytes_recv; };
inline Pending &pending() { static Pending p = {nullptr, nullptr, 0, 0}; return p; }
inline void try_match() {
    Pending &p = pending();
    if (p.send && p.recv) {
        size_t n = p.bytes_send < p.bytes_recv ? p.bytes_send : p.bytes_recv;
        std::memmove(p.recv, p.send, n);
        p.send = nullptr; p.recv = nullptr;
    }
}
}

inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
inline int MPI_Comm_group(MPI_Comm, MPI_Group *g) { *g = 1; return 0; }
inline int MPI_Group_incl(MPI_Group, int, const int *, MPI_Group *g) { *g = 1; return 0; }
inline int MPI_Comm_create_group(MPI_Comm, MPI_Group, int, MPI_Comm *c) { *c = 1; return 0; }
inline int MPI_Group_free(MPI_Group *g) { *g = 0; return 0; }
inline int MPI_Comm_free(MPI_Comm *c) { *c = MPI_COMM_NULL; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Abort(MPI_Comm, int code) { std::exit(code); return 0; }

inline int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype st, int, int,
                        void *rbuf, int rcount, MPI_Datatype rt, int, int, MPI_Comm, MPI_Status *) {
    size_t ns = (size_t)scount * (size_t)st, nr = (size_t)rcount * (size_t)rt;
    std::memmove(rbuf, sbuf, ns < nr ? ns : nr);
    return 0;
}
inline int MPI_Isend(const void *buf, int count, MPI_Datatype t, int, int, MPI_Comm, MPI_Request *req) {
    glac_mpishim::pending().send = buf;
    glac_mpishim::pending().bytes_send = (size_t)count * (size_t)t;
    glac_mpishim::try_match();
    *req = 1;
    return 0;
}
inline int MPI_Irecv(void *buf, int count, MPI_Datatype t, int, int, MPI_Comm, MPI_Request *req) {
    glac_mpishim::pending().recv = buf;
    glac_mpishim::pending().bytes_recv = (size_t)count * (size_t)t;
    glac_mpishim::try_match();
    *req = 2;
    return 0;
}
inline int MPI_Wait(MPI_Request *req, MPI_Status *) { glac_mpishim::try_match(); *req = 0; return 0; }

inline int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (sbuf != rbuf) std::memmove(rbuf, sbuf, (size_t)count * (size_t)t);
    return 0;
}
inline int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    if (sbuf != rbuf) std::memmove(rbuf, sbuf, (size_t)count * (size_t)t);
    return 0;
}
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }

inline int MPI_File_open(MPI_Comm, const char *name, int mode, MPI_Info, MPI_File *fh) {
    int flags = (mode & MPI_MODE_WRONLY) ? O_WRONLY : O_RDONLY;
    if (mode & MPI_MODE_CREATE) flags |= O_CREAT;
    *fh = open(name, flags, 0644);
    return *fh < 0 ? 1 : 0;
}
inline int MPI_File_close(MPI_File *fh) { if (*fh >= 0) close(*fh); *fh = -1; return 0; }
inline int MPI_File_read_at(MPI_File fh, MPI_Offset off, void *buf, int count, MPI_Datatype t, MPI_Status *) {
    ssize_t n = pread(fh, buf, (size_t)count * (size_t)t, (off_t)off);
    return n < 0 ? 1 : 0;
}
inline int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int count, MPI_Datatype t, MPI_Status *) {
    ssize_t n = pwrite(fh, buf, (size_t)count * (size_t)t, (off_t)off);
    return n < 0 ? 1 : 0;
}

#endif
