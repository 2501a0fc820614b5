/*
 * Single-rank MPI subset -- TEST INFRASTRUCTURE ONLY (oracle build).
 * See mpi.h for scope.  Every collective degenerates to a local copy
 * (pack with the send datatype, unpack with the receive datatype), which is
 * what OpenMPI does for a communicator of size one.
 */
#include "mpi.h"

#include <setjmp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

struct shim_dtype {
    size_t elem;        /* bytes of one basic unit addressed by the subarray */
    int nd;             /* 0 = contiguous unit, else subarray rank */
    int sizes[4], subsizes[4], starts[4];
    int predefined;
};

struct shim_dtype shim_mpi_double = {sizeof(double), 0, {0}, {0}, {0}, 1};
struct shim_dtype shim_mpi_int = {sizeof(int), 0, {0}, {0}, {0}, 1};
struct shim_dtype shim_mpi_char = {1, 0, {0}, {0}, {0}, 1};

/* Optional escape hatch: when set, MPI_Abort longjmps here instead of
 * terminating the process (used by the oracle driver's ctypes entry points). */
jmp_buf *shim_abort_target = NULL;

static size_t dt_extent(MPI_Datatype t)
{
    size_t n = t->elem;
    for (int d = 0; d < t->nd; d++) n *= (size_t) t->sizes[d];
    return n;
}

static size_t dt_size(MPI_Datatype t)
{
    size_t n = t->elem;
    for (int d = 0; d < t->nd; d++) n *= (size_t) t->subsizes[d];
    return n;
}

/* Visit every contiguous run of a datatype instance: callback(offset, bytes). */
typedef void (*run_fn)(size_t off, size_t len, void *ctx);

static void dt_runs(MPI_Datatype t, run_fn fn, void *ctx)
{
    if (t->nd == 0) {
        fn(0, t->elem, ctx);
        return;
    }
    int nd = t->nd;
    size_t run = (size_t) t->subsizes[nd - 1] * t->elem;
    size_t stride[4];
    stride[nd - 1] = t->elem;
    for (int d = nd - 2; d >= 0; d--) stride[d] = stride[d + 1] * (size_t) t->sizes[d + 1];
    int idx[4] = {0, 0, 0, 0};
    size_t nouter = 1;
    for (int d = 0; d < nd - 1; d++) nouter *= (size_t) t->subsizes[d];
    if (run == 0) return;
    for (size_t o = 0; o < nouter; o++) {
        size_t off = (size_t) t->starts[nd - 1] * stride[nd - 1];
        for (int d = 0; d < nd - 1; d++) off += (size_t) (t->starts[d] + idx[d]) * stride[d];
        fn(off, run, ctx);
        for (int d = nd - 2; d >= 0; d--) {
            if (++idx[d] < t->subsizes[d]) break;
            idx[d] = 0;
        }
    }
}

struct copy_ctx { char *base; char *buf; size_t pos; int to_buf; };

static void copy_run(size_t off, size_t len, void *vctx)
{
    struct copy_ctx *c = (struct copy_ctx *) vctx;
    if (c->to_buf) memcpy(c->buf + c->pos, c->base + off, len);
    else memcpy(c->base + off, c->buf + c->pos, len);
    c->pos += len;
}

static size_t pack(const void *src, int count, MPI_Datatype t, char *dst)
{
    struct copy_ctx c = {NULL, dst, 0, 1};
    for (int i = 0; i < count; i++) {
        c.base = (char *) src + (size_t) i * dt_extent(t);
        dt_runs(t, copy_run, &c);
    }
    return c.pos;
}

static size_t unpack(void *dst, int count, MPI_Datatype t, const char *src)
{
    struct copy_ctx c = {NULL, (char *) src, 0, 0};
    for (int i = 0; i < count; i++) {
        c.base = (char *) dst + (size_t) i * dt_extent(t);
        dt_runs(t, copy_run, &c);
    }
    return c.pos;
}

int MPI_Init(int *argc, char ***argv) { (void) argc; (void) argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Initialized(int *flag) { *flag = 1; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void) comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void) comm; *size = 1; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm comm) { (void) comm; return MPI_SUCCESS; }

int MPI_Abort(MPI_Comm comm, int errorcode)
{
    (void) comm;
    fflush(stdout);
    fflush(stderr);
    if (shim_abort_target) longjmp(*shim_abort_target, errorcode ? errorcode : 1);
    exit(errorcode);
}

int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[], const int periods[],
                    int reorder, MPI_Comm *comm_cart)
{
    (void) old; (void) periods; (void) reorder;
    for (int d = 0; d < ndims; d++)
        if (dims[d] != 1) {
            fprintf(stderr, "mpi shim: Cartesian grid must be 1x..x1 at one rank\n");
            MPI_Abort(0, 1);
        }
    *comm_cart = 1;
    return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[])
{
    (void) comm; (void) rank;
    for (int d = 0; d < maxdims; d++) coords[d] = 0;
    return MPI_SUCCESS;
}

int MPI_Cart_rank(MPI_Comm comm, const int coords[], int *rank)
{
    (void) comm; (void) coords;
    *rank = 0;
    return MPI_SUCCESS;
}

int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *src, int *dst)
{
    (void) comm; (void) direction; (void) disp;
    *src = 0;
    *dst = 0;
    return MPI_SUCCESS;
}

int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype *newtype)
{
    if (oldtype->nd != 0) return MPI_ERR_OTHER;
    MPI_Datatype t = (MPI_Datatype) calloc(1, sizeof(*t));
    t->elem = oldtype->elem * (size_t) count;
    *newtype = t;
    return MPI_SUCCESS;
}

int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[],
                             const int starts[], int order, MPI_Datatype oldtype,
                             MPI_Datatype *newtype)
{
    if (oldtype->nd != 0 || ndims < 1 || ndims > 4) return MPI_ERR_OTHER;
    MPI_Datatype t = (MPI_Datatype) calloc(1, sizeof(*t));
    t->elem = oldtype->elem;
    t->nd = ndims;
    for (int d = 0; d < ndims; d++) {
        int s = order == MPI_ORDER_C ? d : ndims - 1 - d;
        t->sizes[d] = sizes[s];
        t->subsizes[d] = subsizes[s];
        t->starts[d] = starts[s];
        if (starts[s] < 0 || subsizes[s] < 0 || starts[s] + subsizes[s] > sizes[s]) {
            fprintf(stderr, "mpi shim: subarray out of range\n");
            free(t);
            return MPI_ERR_OTHER;
        }
    }
    *newtype = t;
    return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype *type) { (void) type; return MPI_SUCCESS; }

int MPI_Type_free(MPI_Datatype *type)
{
    if (*type && !(*type)->predefined) free(*type);
    *type = NULL;
    return MPI_SUCCESS;
}

int MPI_Alltoallw(const void *sendbuf, const int sendcounts[], const int sdispls[],
                  const MPI_Datatype sendtypes[], void *recvbuf, const int recvcounts[],
                  const int rdispls[], const MPI_Datatype recvtypes[], MPI_Comm comm)
{
    (void) comm;
    size_t ns = (size_t) sendcounts[0] * dt_size(sendtypes[0]);
    size_t nr = (size_t) recvcounts[0] * dt_size(recvtypes[0]);
    if (ns != nr) {
        fprintf(stderr, "mpi shim: Alltoallw size mismatch %zu != %zu\n", ns, nr);
        MPI_Abort(0, 1);
    }
    if (ns == 0) return MPI_SUCCESS;
    char *tmp = (char *) malloc(ns);
    pack((const char *) sendbuf + sdispls[0], sendcounts[0], sendtypes[0], tmp);
    unpack((char *) recvbuf + rdispls[0], recvcounts[0], recvtypes[0], tmp);
    free(tmp);
    return MPI_SUCCESS;
}

/* Point-to-point to self: Isend packs into a FIFO, Recv unpacks the oldest
 * message with the matching tag. */
struct shim_msg { int tag; size_t n; char *data; struct shim_msg *next; };
static struct shim_msg *msg_head = NULL;
struct shim_request { int done; };

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *request)
{
    (void) dest; (void) comm;
    struct shim_msg *m = (struct shim_msg *) malloc(sizeof(*m));
    m->tag = tag;
    m->n = (size_t) count * dt_size(type);
    m->data = (char *) malloc(m->n ? m->n : 1);
    pack(buf, count, type, m->data);
    m->next = NULL;
    struct shim_msg **pp = &msg_head;
    while (*pp) pp = &(*pp)->next;
    *pp = m;
    *request = (MPI_Request) calloc(1, sizeof(struct shim_request));
    (*request)->done = 1;
    return MPI_SUCCESS;
}

int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag,
             MPI_Comm comm, MPI_Status *status)
{
    (void) source; (void) comm;
    struct shim_msg **pp = &msg_head;
    while (*pp && (*pp)->tag != tag) pp = &(*pp)->next;
    if (!*pp) {
        fprintf(stderr, "mpi shim: Recv with no matching send (tag %d)\n", tag);
        MPI_Abort(0, 1);
    }
    struct shim_msg *m = *pp;
    if (m->n != (size_t) count * dt_size(type)) {
        fprintf(stderr, "mpi shim: Recv size mismatch\n");
        MPI_Abort(0, 1);
    }
    unpack(buf, count, type, m->data);
    *pp = m->next;
    free(m->data);
    free(m);
    if (status) { status->MPI_SOURCE = 0; status->MPI_TAG = tag; status->MPI_ERROR = 0; }
    return MPI_SUCCESS;
}

int MPI_Wait(MPI_Request *request, MPI_Status *status)
{
    (void) status;
    free(*request);
    *request = NULL;
    return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                  MPI_Op op, MPI_Comm comm)
{
    (void) op; (void) comm;
    if (sendbuf != MPI_IN_PLACE) memcpy(recvbuf, sendbuf, (size_t) count * dt_size(type));
    return MPI_SUCCESS;
}

int MPI_Gather(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
               void *recvbuf, int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm)
{
    (void) recvcount; (void) recvtype; (void) root; (void) comm;
    if (sendbuf != MPI_IN_PLACE) memcpy(recvbuf, sendbuf, (size_t) sendcount * dt_size(sendtype));
    return MPI_SUCCESS;
}

int MPI_Gatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                void *recvbuf, const int recvcounts[], const int displs[],
                MPI_Datatype recvtype, int root, MPI_Comm comm)
{
    (void) recvcounts; (void) root; (void) comm;
    memcpy((char *) recvbuf + (size_t) displs[0] * dt_extent(recvtype), sendbuf,
           (size_t) sendcount * dt_size(sendtype));
    return MPI_SUCCESS;
}

/* MPI-IO through stdio.  A view is (displacement, filetype); the filetype is
 * tiled along the file, as in MPI. */
struct shim_file {
    FILE *fp;
    char *name;
    int delete_on_close;
    MPI_Offset disp;
    MPI_Datatype filetype;
};

int MPI_File_open(MPI_Comm comm, const char *filename, int amode, MPI_Info info, MPI_File *fh)
{
    (void) comm; (void) info;
    FILE *fp = NULL;
    int exists = access(filename, F_OK) == 0;
    if (amode & MPI_MODE_RDONLY) {
        fp = fopen(filename, "rb");
    } else {
        if ((amode & MPI_MODE_EXCL) && exists) return MPI_ERR_OTHER;
        if (!exists && !(amode & MPI_MODE_CREATE)) return MPI_ERR_OTHER;
        fp = exists ? fopen(filename, "r+b") : fopen(filename, "w+b");
    }
    if (!fp) return MPI_ERR_OTHER;
    MPI_File f = (MPI_File) calloc(1, sizeof(*f));
    f->fp = fp;
    f->name = strdup(filename);
    f->delete_on_close = (amode & MPI_MODE_DELETE_ON_CLOSE) != 0;
    f->disp = 0;
    f->filetype = MPI_CHAR;
    *fh = f;
    return MPI_SUCCESS;
}

int MPI_File_close(MPI_File *fh)
{
    MPI_File f = *fh;
    fclose(f->fp);
    if (f->delete_on_close) remove(f->name);
    free(f->name);
    free(f);
    *fh = NULL;
    return MPI_SUCCESS;
}

int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype,
                      MPI_Datatype filetype, const char *datarep, MPI_Info info)
{
    (void) etype; (void) datarep; (void) info;
    fh->disp = disp;
    fh->filetype = filetype;
    return MPI_SUCCESS;
}

struct file_ctx { MPI_File f; char *buf; size_t pos, total; MPI_Offset base; int writing; int err; };

static void file_run(size_t off, size_t len, void *vctx)
{
    struct file_ctx *c = (struct file_ctx *) vctx;
    if (c->pos >= c->total || c->err) return;
    if (len > c->total - c->pos) len = c->total - c->pos;
    if (fseeko(c->f->fp, (off_t) (c->base + (MPI_Offset) off), SEEK_SET) != 0) { c->err = 1; return; }
    size_t n = c->writing ? fwrite(c->buf + c->pos, 1, len, c->f->fp)
                          : fread(c->buf + c->pos, 1, len, c->f->fp);
    if (n != len) c->err = 1;
    c->pos += len;
}

static int file_xfer(MPI_File fh, char *bytes, size_t total, int writing)
{
    struct file_ctx c = {fh, bytes, 0, total, fh->disp, writing, 0};
    size_t ext = dt_extent(fh->filetype);
    while (c.pos < c.total && !c.err) {
        dt_runs(fh->filetype, file_run, &c);
        c.base += (MPI_Offset) ext;
    }
    return c.err ? MPI_ERR_OTHER : MPI_SUCCESS;
}

int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype type,
                       MPI_Status *status)
{
    (void) status;
    size_t n = (size_t) count * dt_size(type);
    char *tmp = (char *) malloc(n ? n : 1);
    pack(buf, count, type, tmp);
    int rc = file_xfer(fh, tmp, n, 1);
    free(tmp);
    return rc;
}

int MPI_File_read_all(MPI_File fh, void *buf, int count, MPI_Datatype type,
                      MPI_Status *status)
{
    (void) status;
    size_t n = (size_t) count * dt_size(type);
    char *tmp = (char *) malloc(n ? n : 1);
    int rc = file_xfer(fh, tmp, n, 0);
    if (rc == MPI_SUCCESS) unpack(buf, count, type, tmp);
    free(tmp);
    return rc;
}
