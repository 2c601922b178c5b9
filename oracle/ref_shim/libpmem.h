/*
 * Stand-in for libpmem's header, used only to compile the reference's join and generator sources into
 * the CPU baseline under oracle/_ref (libpmem is not installed here). The reference uses libpmem only
 * to map its .bin relation files (src/inc/utils.c:486-520) and for persist/flush calls on NVM; in the
 * DRAM configuration measured here a file mapping is an mmap of the file and persisting is a plain
 * memcpy/memset.
 */
#ifndef HJREF_LIBPMEM_SHIM_H
#define HJREF_LIBPMEM_SHIM_H
#include <fcntl.h>
#include <string.h>
#include <sys/mman.h>
#include <unistd.h>

#define PMEM_FILE_CREATE (1 << 0)
#define PMEM_FILE_EXCL (1 << 1)

static inline void *pmem_map_file(const char *path, size_t len, int flags, int mode, size_t *mapped_lenp,
                                  int *is_pmemp) {
    int oflags = O_RDWR;
    if (flags & PMEM_FILE_CREATE) oflags |= O_CREAT;
    if (flags & PMEM_FILE_EXCL) oflags |= O_EXCL;
    int fd = open(path, oflags, mode);
    if (fd < 0) return NULL;
    /* The size comes from lseek: <sys/stat.h> would clash with the reference's own mkdir(). */
    off_t size = lseek(fd, 0, SEEK_END);
    if (size < 0) { close(fd); return NULL; }
    if ((size_t)size < len && ftruncate(fd, (off_t)len) != 0) { close(fd); return NULL; }
    if (len == 0) len = (size_t)size;
    void *p = mmap(NULL, len, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
    close(fd);
    if (p == MAP_FAILED) return NULL;
    if (mapped_lenp) *mapped_lenp = len;
    if (is_pmemp) *is_pmemp = 1;
    return p;
}
static inline int pmem_unmap(void *addr, size_t len) { return munmap(addr, len); }
static inline void *pmem_memcpy_persist(void *d, const void *s, size_t n) { return memcpy(d, s, n); }
static inline void *pmem_memset_persist(void *d, int c, size_t n) { return memset(d, c, n); }
static inline void pmem_persist(const void *a, size_t n) { (void)a; (void)n; }
static inline int pmem_msync(const void *a, size_t n) { (void)a; (void)n; return 0; }
#endif
