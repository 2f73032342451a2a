/*
 * Single-rank stand-in for <mpi.h>, used ONLY to compile the reference
 * solver's own C++ sources into the CPU oracle binary (oracle/_ref).
 * Test infrastructure: never linked into the product library.
 *
 * Written from the MPI-3.1 standard's semantics for a communicator of size 1:
 *   - every collective is a local copy (or a no-op when in place);
 *   - Cartesian topologies are 1x1; a periodic shift returns rank 0 itself,
 *     a non-periodic shift returns MPI_PROC_NULL;
 *   - MPI-IO views cover the whole file region from `disp` onward, which is
 *     exactly the single-rank case of the subarray views the reference sets.
 * Point-to-point halo exchange is not on the oracle's path; those calls abort.
 */
#ifndef MC3D_ORACLE_MPI_SHIM_H
#define MC3D_ORACLE_MPI_SHIM_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef long long MPI_Offset;
struct MPI_Status { int MPI_SOURCE, MPI_TAG, MPI_ERROR; };
struct mc3d_shim_file { FILE *fp; MPI_Offset view; };
typedef mc3d_shim_file *MPI_File;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_PROC_NULL (-2)
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_ORDER_C 56
#define MPI_ORDER_FORTRAN 57
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_MODE_RDWR 8
#define MPI_MODE_CREATE 1

#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUM 3
#define MPI_LOR 4

/* predefined datatypes are handles into a byte-size registry */
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_DOUBLE 3
#define MPI_DOUBLE_PRECISION 4
#define MPI_C_BOOL 5
#define MPI_FLOAT 6
#define MPI_LONG 7

inline std::vector<long long> &mc3d_shim_types() {
    static std::vector<long long> sizes = {0, 1, 4, 8, 8, (long long)sizeof(bool), 4, (long long)sizeof(long)};
    return sizes;
}
inline long long mc3d_shim_tsize(MPI_Datatype t) {
    std::vector<long long> &s = mc3d_shim_types();
    if (t <= 0 || t >= (int)s.size()) { fprintf(stderr, "mpi shim: bad datatype %d\n", t); abort(); }
    return s[t];
}
inline MPI_Datatype mc3d_shim_newtype(long long bytes) {
    mc3d_shim_types().push_back(bytes);
    return (MPI_Datatype)(mc3d_shim_types().size() - 1);
}

inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Abort(MPI_Comm, int code) {
    fprintf(stderr, "mpi shim: MPI_Abort(%d)\n", code);
    exit(code == 0 ? 1 : (code & 0xff ? code & 0xff : 1));
}
inline double MPI_Wtime() {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }

inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (s != MPI_IN_PLACE && s != r) memcpy(r, s, (size_t)(n * mc3d_shim_tsize(t)));
    return MPI_SUCCESS;
}
inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int, MPI_Comm c) {
    return MPI_Allreduce(s, r, n, t, op, c);
}

inline int MPI_Alltoallv(const void *s, const int *scnt, const int *sdsp, MPI_Datatype st,
                         void *r, const int *rcnt, const int *rdsp, MPI_Datatype rt, MPI_Comm) {
    long long sb = mc3d_shim_tsize(st), rb = mc3d_shim_tsize(rt);
    if (scnt[0] * sb != rcnt[0] * rb) { fprintf(stderr, "mpi shim: alltoallv size mismatch\n"); abort(); }
    memmove((char *)r + rdsp[0] * rb, (const char *)s + sdsp[0] * sb, (size_t)(scnt[0] * sb));
    return MPI_SUCCESS;
}
inline int MPI_Ialltoallv(const void *s, const int *scnt, const int *sdsp, MPI_Datatype st,
                          void *r, const int *rcnt, const int *rdsp, MPI_Datatype rt, MPI_Comm c,
                          MPI_Request *req) {
    *req = 0;
    return MPI_Alltoallv(s, scnt, sdsp, st, r, rcnt, rdsp, rt, c);
}
inline int MPI_Wait(MPI_Request *, MPI_Status *) { return MPI_SUCCESS; }
inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return MPI_SUCCESS; }
inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
    fprintf(stderr, "mpi shim: point-to-point halo exchange is not supported\n"); abort();
}
inline int MPI_Issend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
    fprintf(stderr, "mpi shim: point-to-point halo exchange is not supported\n"); abort();
}

/* Cartesian topology: remember the periodic flags of each communicator */
inline std::vector<std::vector<int> > &mc3d_shim_carts() {
    static std::vector<std::vector<int> > c(1, std::vector<int>(3, 0));
    return c;
}
inline int MPI_Cart_create(MPI_Comm, int nd, const int *dims, const int *per, int, MPI_Comm *out) {
    for (int i = 0; i < nd; i++)
        if (dims[i] != 1 && dims[i] != 0) { fprintf(stderr, "mpi shim: only 1x1 grids\n"); abort(); }
    std::vector<int> p(3, 0);
    for (int i = 0; i < nd && i < 3; i++) p[i] = per[i];
    mc3d_shim_carts().push_back(p);
    *out = (MPI_Comm)(mc3d_shim_carts().size() - 1);
    return MPI_SUCCESS;
}
inline int MPI_Cart_coords(MPI_Comm, int, int nd, int *coords) {
    for (int i = 0; i < nd; i++) coords[i] = 0;
    return MPI_SUCCESS;
}
inline int MPI_Cart_sub(MPI_Comm c, const int *, MPI_Comm *out) {
    mc3d_shim_carts().push_back(mc3d_shim_carts()[c < 0 ? 0 : c]);
    *out = (MPI_Comm)(mc3d_shim_carts().size() - 1);
    return MPI_SUCCESS;
}
inline int MPI_Cart_shift(MPI_Comm c, int dir, int, int *src, int *dst) {
    int per = (c >= 0 && c < (int)mc3d_shim_carts().size() && dir < 3) ? mc3d_shim_carts()[c][dir] : 0;
    *src = *dst = per ? 0 : MPI_PROC_NULL;
    return MPI_SUCCESS;
}

/* derived datatypes: only their byte size matters for one rank */
inline int MPI_Type_size(MPI_Datatype t, int *sz) { *sz = (int)mc3d_shim_tsize(t); return MPI_SUCCESS; }
inline int MPI_Type_contiguous(int n, MPI_Datatype t, MPI_Datatype *o) {
    *o = mc3d_shim_newtype(n * mc3d_shim_tsize(t)); return MPI_SUCCESS;
}
inline int MPI_Type_vector(int n, int bl, int, MPI_Datatype t, MPI_Datatype *o) {
    *o = mc3d_shim_newtype((long long)n * bl * mc3d_shim_tsize(t)); return MPI_SUCCESS;
}
inline int MPI_Type_create_subarray(int nd, const int *, const int *sub, const int *, int,
                                    MPI_Datatype t, MPI_Datatype *o) {
    long long n = 1;
    for (int i = 0; i < nd; i++) n *= sub[i];
    *o = mc3d_shim_newtype(n * mc3d_shim_tsize(t)); return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype *t) { *t = 0; return MPI_SUCCESS; }

/* MPI-IO for one rank: a view starts at byte `disp` and is contiguous */
inline int MPI_File_open(MPI_Comm, const char *name, int mode, MPI_Info, MPI_File *fh) {
    const char *m = (mode & MPI_MODE_RDONLY) ? "rb" : "r+b";
    FILE *fp = fopen(name, m);
    if (!fp && (mode & MPI_MODE_CREATE)) fp = fopen(name, "w+b");
    if (!fp) { fprintf(stderr, "mpi shim: cannot open %s\n", name); *fh = 0; return 1; }
    *fh = new mc3d_shim_file{fp, 0};
    return MPI_SUCCESS;
}
inline int MPI_File_close(MPI_File *fh) {
    if (*fh) { fclose((*fh)->fp); delete *fh; *fh = 0; }
    return MPI_SUCCESS;
}
inline int MPI_File_set_size(MPI_File, MPI_Offset) { return MPI_SUCCESS; }
inline int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype, MPI_Datatype, const char *, MPI_Info) {
    fh->view = disp; return MPI_SUCCESS;
}
inline int MPI_File_write_all(MPI_File fh, const void *buf, int n, MPI_Datatype t, MPI_Status *) {
    fseeko(fh->fp, (off_t)fh->view, SEEK_SET);
    size_t b = (size_t)(n * mc3d_shim_tsize(t));
    if (fwrite(buf, 1, b, fh->fp) != b) return 1;
    fh->view += (MPI_Offset)b;
    return MPI_SUCCESS;
}
inline int MPI_File_read_all(MPI_File fh, void *buf, int n, MPI_Datatype t, MPI_Status *) {
    fseeko(fh->fp, (off_t)fh->view, SEEK_SET);
    size_t b = (size_t)(n * mc3d_shim_tsize(t));
    if (fread(buf, 1, b, fh->fp) != b) return 1;
    fh->view += (MPI_Offset)b;
    return MPI_SUCCESS;
}
inline int MPI_File_write_at_all(MPI_File fh, MPI_Offset off, const void *buf, int n, MPI_Datatype t, MPI_Status *s) {
    fh->view = off; return MPI_File_write_all(fh, buf, n, t, s);
}
inline int MPI_File_read_at_all(MPI_File fh, MPI_Offset off, void *buf, int n, MPI_Datatype t, MPI_Status *s) {
    fh->view = off; return MPI_File_read_all(fh, buf, n, t, s);
}
inline int MPI_File_write(MPI_File fh, const void *buf, int n, MPI_Datatype t, MPI_Status *s) {
    return MPI_File_write_all(fh, buf, n, t, s);
}
inline int MPI_File_read(MPI_File fh, void *buf, int n, MPI_Datatype t, MPI_Status *s) {
    return MPI_File_read_all(fh, buf, n, t, s);
}
inline int MPI_File_get_size(MPI_File fh, MPI_Offset *sz) {
    off_t cur = ftello(fh->fp); fseeko(fh->fp, 0, SEEK_END);
    *sz = (MPI_Offset)ftello(fh->fp); fseeko(fh->fp, cur, SEEK_SET);
    return MPI_SUCCESS;
}
inline int MPI_File_seek(MPI_File fh, MPI_Offset off, int) { fh->view = off; return MPI_SUCCESS; }
#define MPI_SEEK_SET 600

#endif
