/* Shared state of the drop-in libraries: one context on HH_DEVICE (default 0), one cached plan
 * keyed by the problem's sizes and stencil bytes, and staging buffers that grow on demand and are
 * kept for the life of the process (the reference's entry points are called in loops; they
 * should not pay a device allocation per call). */
#ifndef HH_DROPIN_COMMON_H
#define HH_DROPIN_COMMON_H

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hh.h"

static hh_ctx  *g_ctx;
static hh_plan *g_plan;
static uint64_t g_key;
static unsigned char *g_keybytes; /* the bytes g_key was made from: a hash hit is confirmed by them */
static size_t   g_keylen;
static int      g_status;
static void    *g_dev_a, *g_dev_b; /* device staging, g_dev_bytes each */
static size_t   g_dev_bytes;
static void    *g_host_tmp;        /* host staging (transposes, real <-> complex planes) */
static size_t   g_host_bytes;

static uint64_t fnv1a(uint64_t h, const void *p, size_t n) {
    const unsigned char *b = (const unsigned char *)p;
    for (size_t i = 0; i < n; i++) {
        h ^= b[i];
        h *= 1099511628211ULL;
    }
    return h;
}

static int report(int rc, const char *what) {
    g_status = rc;
    if (rc != HH_OK) fprintf(stderr, "ERROR: %s failed with %d: %s\n", what, rc, hh_last_error());
    return rc;
}

static hh_ctx *context(void) {
    if (!g_ctx) {
        const char *d = getenv("HH_DEVICE");
        if (report(hh_ctx_create(d ? atoi(d) : 0, NULL, &g_ctx), "hh_ctx_create") != HH_OK) g_ctx = NULL;
    }
    return g_ctx;
}

/* The plan key: `nparts` byte ranges concatenated.  Returns 1 when it equals the cached plan's
 * key (hash and bytes), else makes it the pending key (g_key / g_keybytes) and returns 0; the
 * caller then builds a new plan, or calls key_forget() if that fails. */
static int key_matches(const void *const *parts, const size_t *lens, int nparts) {
    size_t len = 0;
    for (int t = 0; t < nparts; t++) len += lens[t];
    unsigned char *buf = (unsigned char *)malloc(len ? len : 1);
    if (!buf) return 0;
    uint64_t h = 1469598103934665603ULL;
    size_t   off = 0;
    for (int t = 0; t < nparts; t++) {
        memcpy(buf + off, parts[t], lens[t]);
        off += lens[t];
    }
    h = fnv1a(h, buf, len);
    if (g_plan && h == g_key && len == g_keylen && memcmp(buf, g_keybytes, len) == 0) {
        free(buf);
        return 1;
    }
    free(g_keybytes);
    g_keybytes = buf;
    g_keylen = len;
    g_key = h;
    return 0;
}

static void key_forget(void) {
    free(g_keybytes);
    g_keybytes = NULL;
    g_keylen = 0;
    g_key = 0;
}

/* two device buffers of at least `bytes` each (kept and reused) */
static int device_staging(size_t bytes, void **a, void **b) {
    hh_ctx *c = context();
    if (!c) return HH_ERR_CUDA;
    if (g_dev_bytes < bytes) {
        if (g_dev_a) hh_free(c, g_dev_a);
        if (g_dev_b) hh_free(c, g_dev_b);
        g_dev_a = g_dev_b = NULL;
        g_dev_bytes = 0;
        int rc = hh_malloc(c, bytes, &g_dev_a);
        if (rc == HH_OK) rc = hh_malloc(c, bytes, &g_dev_b);
        if (rc != HH_OK) {
            if (g_dev_a) hh_free(c, g_dev_a);
            g_dev_a = NULL;
            return rc;
        }
        g_dev_bytes = bytes;
    }
    *a = g_dev_a;
    *b = g_dev_b;
    return HH_OK;
}

/* a host buffer of at least `bytes` (kept and reused) */
static void *host_staging(size_t bytes) {
    if (g_host_bytes < bytes) {
        free(g_host_tmp);
        g_host_tmp = malloc(bytes);
        g_host_bytes = g_host_tmp ? bytes : 0;
    }
    return g_host_tmp;
}

#endif
