/* Shared state of the drop-in libraries: one context on HH_DEVICE (default 0) and one cached
 * plan keyed by the problem's sizes and stencil bytes. */
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
static int      g_status;

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

/* device round trip of `count` complex values through `fn` (a device-side transform) */
static int device_staging(size_t bytes, void **a, void **b) {
    hh_ctx *c = context();
    if (!c) return HH_ERR_CUDA;
    *a = *b = NULL;
    int rc = hh_malloc(c, bytes, a);
    if (rc == HH_OK) rc = hh_malloc(c, bytes, b);
    if (rc != HH_OK) {
        if (*a) hh_free(c, *a);
        *a = NULL;
    }
    return rc;
}

#endif
