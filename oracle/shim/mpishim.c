/*
 * Single-rank MPI shim (test infrastructure, see mpi.h).  Every call acts as
 * if MPI_COMM_WORLD held one process: messages a rank sends to itself are
 * packed from the send layout and unpacked into the receive layout.
 */
#include "mpi.h"

#include <stdlib.h>
#include <string.h>

struct oracle_mpi_type {
    int kind;            /* 0 basic, 1 subarray, 2 contiguous */
    size_t elem;         /* bytes of one basic element */
    int ndims;
    int sizes[8], subsizes[8], starts[8];
    int count;           /* contiguous: number of old elements */
    struct oracle_mpi_type *old;
};

struct oracle_mpi_type oracle_mpi_double = {0, sizeof(double)};
struct oracle_mpi_type oracle_mpi_int = {0, sizeof(int)};
struct oracle_mpi_type oracle_mpi_uchar = {0, sizeof(unsigned char)};
struct oracle_mpi_type oracle_mpi_ushort = {0, sizeof(unsigned short)};
struct oracle_mpi_type oracle_mpi_unsigned = {0, sizeof(unsigned)};
struct oracle_mpi_type oracle_mpi_ulong = {0, sizeof(unsigned long)};
struct oracle_mpi_type oracle_mpi_ulonglong = {0, sizeof(unsigned long long)};

struct oracle_mpi_file {
    FILE *fp;
    MPI_Offset disp;
    MPI_Datatype filetype;
};

/* number of basic elements one item of `t` carries */
static size_t type_elems(MPI_Datatype t)
{
    if (t->kind == 0) return 1;
    if (t->kind == 2) return (size_t)t->count * type_elems(t->old);
    size_t n = 1;
    for (int d = 0; d < t->ndims; d++) n *= (size_t)t->subsizes[d];
    return n * type_elems(t->old);
}

/* extent in bytes of one item of `t` (subarray: the whole enclosing array) */
static size_t type_extent(MPI_Datatype t)
{
    if (t->kind == 0) return t->elem;
    if (t->kind == 2) return (size_t)t->count * type_extent(t->old);
    size_t n = 1;
    for (int d = 0; d < t->ndims; d++) n *= (size_t)t->sizes[d];
    return n * type_extent(t->old);
}

/* Walk the byte offsets (relative to the item start) of every basic element
 * of one item of `t`, in type-map order, calling fn(offset). */
typedef void (*visit_fn)(size_t off, size_t elem, void *ctx);

static void visit(MPI_Datatype t, size_t base, visit_fn fn, void *ctx)
{
    if (t->kind == 0) { fn(base, t->elem, ctx); return; }
    if (t->kind == 2) {
        size_t ext = type_extent(t->old);
        for (int i = 0; i < t->count; i++) visit(t->old, base + i * ext, fn, ctx);
        return;
    }
    /* C-order subarray */
    size_t ext = type_extent(t->old);
    int idx[8] = {0};
    size_t total = 1;
    for (int d = 0; d < t->ndims; d++) total *= (size_t)t->subsizes[d];
    for (size_t n = 0; n < total; n++) {
        size_t lin = 0;
        for (int d = 0; d < t->ndims; d++)
            lin = lin * (size_t)t->sizes[d] + (size_t)(t->starts[d] + idx[d]);
        visit(t->old, base + lin * ext, fn, ctx);
        for (int d = t->ndims - 1; d >= 0; d--) {
            if (++idx[d] < t->subsizes[d]) break;
            idx[d] = 0;
        }
    }
}

struct pack_ctx { const char *src; char *dst; size_t pos; };

static void pack_one(size_t off, size_t elem, void *c)
{
    struct pack_ctx *p = (struct pack_ctx *)c;
    memcpy(p->dst + p->pos, p->src + off, elem);
    p->pos += elem;
}

static void unpack_one(size_t off, size_t elem, void *c)
{
    struct pack_ctx *p = (struct pack_ctx *)c;
    memcpy(p->dst + off, p->src + p->pos, elem);
    p->pos += elem;
}

static char *pack(const void *buf, int count, MPI_Datatype t, size_t *nbytes)
{
    size_t n = (size_t)count * type_elems(t) * 16 + 16;
    char *out = (char *)malloc(n);
    struct pack_ctx c = {(const char *)buf, out, 0};
    size_t ext = type_extent(t);
    for (int i = 0; i < count; i++) visit(t, (size_t)i * ext, pack_one, &c);
    *nbytes = c.pos;
    return out;
}

static void unpack(const char *bytes, void *buf, int count, MPI_Datatype t)
{
    struct pack_ctx c = {bytes, (char *)buf, 0};
    size_t ext = type_extent(t);
    for (int i = 0; i < count; i++) visit(t, (size_t)i * ext, unpack_one, &c);
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm)
{
    (void)buf; (void)count; (void)type; (void)root; (void)comm;
    return MPI_SUCCESS; /* the root's buffer is already everyone's buffer */
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype type, MPI_Op op, MPI_Comm comm)
{
    (void)op; (void)comm; /* MIN/MAX over one contribution is that value */
    if (sendbuf != recvbuf) memmove(recvbuf, sendbuf, (size_t)count * type_extent(type));
    return MPI_SUCCESS;
}

int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                 int dest, int sendtag, void *recvbuf, int recvcount,
                 MPI_Datatype recvtype, int source, int recvtag, MPI_Comm comm,
                 MPI_Status *status)
{
    (void)dest; (void)sendtag; (void)source; (void)recvtag; (void)comm;
    size_t nbytes;
    char *bytes = pack(sendbuf, sendcount, sendtype, &nbytes);
    /* a basic receive type takes as many elements as were sent (at most
     * recvcount, as MPI requires the buffer to be large enough) */
    int n = recvcount;
    if (recvtype->kind == 0 && (size_t)n * recvtype->elem > nbytes)
        n = (int)(nbytes / recvtype->elem);
    unpack(bytes, recvbuf, n, recvtype);
    free(bytes);
    if (status) { status->source = 0; status->tag = 0; status->error = 0; }
    return MPI_SUCCESS;
}

/* Self-addressed messages for MPI_Send/MPI_Recv: a FIFO queue. */
struct msg { char *bytes; size_t n; struct msg *next; };
static struct msg *q_head = NULL, *q_tail = NULL;

int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag,
             MPI_Comm comm)
{
    (void)dest; (void)tag; (void)comm;
    struct msg *m = (struct msg *)malloc(sizeof *m);
    m->bytes = pack(buf, count, type, &m->n);
    m->next = NULL;
    if (q_tail) q_tail->next = m; else q_head = m;
    q_tail = m;
    return MPI_SUCCESS;
}

int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag,
             MPI_Comm comm, MPI_Status *status)
{
    (void)source; (void)tag; (void)comm; (void)count;
    if (status) { status->source = 0; status->tag = 0; status->error = 0; }
    struct msg *m = q_head;
    if (!m) return MPI_SUCCESS; /* nothing was sent: the buffer stays as is */
    q_head = m->next;
    if (!q_head) q_tail = NULL;
    unpack(m->bytes, buf, type->kind == 0 ? (int)(m->n / type->elem) : 1, type);
    free(m->bytes);
    free(m);
    return MPI_SUCCESS;
}

int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[],
                             const int starts[], int order, MPI_Datatype old,
                             MPI_Datatype *newtype)
{
    (void)order; /* the reference only uses MPI_ORDER_C */
    struct oracle_mpi_type *t = (struct oracle_mpi_type *)calloc(1, sizeof *t);
    t->kind = 1;
    t->elem = old->elem;
    t->ndims = ndims;
    for (int d = 0; d < ndims; d++) {
        t->sizes[d] = sizes[d];
        t->subsizes[d] = subsizes[d];
        t->starts[d] = starts[d];
    }
    t->old = old;
    *newtype = t;
    return MPI_SUCCESS;
}

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newtype)
{
    struct oracle_mpi_type *t = (struct oracle_mpi_type *)calloc(1, sizeof *t);
    t->kind = 2;
    t->elem = old->elem;
    t->count = count;
    t->old = old;
    *newtype = t;
    return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype *type) { (void)type; return MPI_SUCCESS; }

int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info,
                  MPI_File *fh)
{
    (void)comm; (void)amode; (void)info;
    FILE *fp = fopen(name, "r+b");
    if (!fp) fp = fopen(name, "w+b");
    if (!fp) return 1;
    struct oracle_mpi_file *f = (struct oracle_mpi_file *)calloc(1, sizeof *f);
    f->fp = fp;
    f->filetype = NULL;
    *fh = f;
    return MPI_SUCCESS;
}

int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype,
                      MPI_Datatype filetype, const char *datarep, MPI_Info info)
{
    (void)etype; (void)datarep; (void)info;
    fh->disp = disp;
    fh->filetype = filetype;
    return MPI_SUCCESS;
}

struct fwrite_ctx { FILE *fp; MPI_Offset disp; const char *src; size_t pos; };

static void write_one(size_t off, size_t elem, void *c)
{
    struct fwrite_ctx *w = (struct fwrite_ctx *)c;
    fseek(w->fp, (long)(w->disp + (MPI_Offset)off), SEEK_SET);
    fwrite(w->src + w->pos, 1, elem, w->fp);
    w->pos += elem;
}

int MPI_File_write_all(MPI_File fh, const void *buf, int count,
                       MPI_Datatype type, MPI_Status *status)
{
    (void)status;
    size_t nbytes;
    char *bytes = pack(buf, count, type, &nbytes);
    MPI_Datatype ft = fh->filetype ? fh->filetype : type;
    if (ft->kind == 0) {
        fseek(fh->fp, (long)fh->disp, SEEK_SET);
        fwrite(bytes, 1, nbytes, fh->fp);
    } else {
        /* tile the file type until every packed byte has a place */
        struct fwrite_ctx w = {fh->fp, fh->disp, bytes, 0};
        size_t ext = type_extent(ft);
        for (size_t i = 0; w.pos < nbytes; i++) visit(ft, i * ext, write_one, &w);
    }
    free(bytes);
    return MPI_SUCCESS;
}

int MPI_File_close(MPI_File *fh)
{
    if (fh && *fh) {
        fclose((*fh)->fp);
        free(*fh);
        *fh = NULL;
    }
    return MPI_SUCCESS;
}
