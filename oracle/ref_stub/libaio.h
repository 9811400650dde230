/*
 * Synchronous stand-in for the five libaio entry points that the G-Store
 * reference (gstore.cpp, io_driver) calls.  It exists only so that the
 * reference can be compiled from its own sources on a machine without the
 * libaio headers; it is part of the oracle (test infrastructure), never of
 * the product.
 *
 *   io_setup      -> records nothing, returns 0
 *   io_prep_pread -> fills the control block
 *   io_submit     -> performs every pread immediately (blocking)
 *   io_getevents  -> reports min_nr completions, since all reads finished
 *
 * Reads issued by the reference use O_DIRECT with 512-byte aligned offsets
 * and sizes (gstore.cpp:3050, 3724-3733); pread honours that unchanged.
 */
#ifndef ORACLE_LIBAIO_STUB_H
#define ORACLE_LIBAIO_STUB_H

#include <stddef.h>
#include <unistd.h>

typedef struct oracle_io_ctx* io_context_t;

struct iocb {
    int fd;
    void* buf;
    size_t nbytes;
    long long offset;
};

struct io_event {
    void* data;
    struct iocb* obj;
    long res;
    long res2;
};

static inline int io_setup(int maxevents, io_context_t* ctxp)
{
    (void)maxevents;
    *ctxp = 0;
    return 0;
}

static inline void io_prep_pread(struct iocb* cb, int fd, void* buf,
                                 size_t count, long long offset)
{
    cb->fd = fd;
    cb->buf = buf;
    cb->nbytes = count;
    cb->offset = offset;
}

static inline int io_submit(io_context_t ctx, long nr, struct iocb** ios)
{
    (void)ctx;
    for (long k = 0; k < nr; ++k) {
        struct iocb* cb = ios[k];
        char* dst = (char*)cb->buf;
        size_t left = cb->nbytes;
        long long off = cb->offset;
        while (left > 0) {
            ssize_t got = pread(cb->fd, dst, left, off);
            if (got <= 0) break; /* short read at end of file: rest stays */
            dst += got;
            off += got;
            left -= (size_t)got;
        }
    }
    return (int)nr;
}

static inline int io_getevents(io_context_t ctx, long min_nr, long nr,
                               struct io_event* events, void* timeout)
{
    (void)ctx; (void)nr; (void)events; (void)timeout;
    return (int)min_nr;
}

#endif
