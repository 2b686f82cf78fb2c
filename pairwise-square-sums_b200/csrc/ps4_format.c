/*
 * ps4_format.c -- result-line text of the C-ABI, byte-identical to the reference's
 * output (exhaustive/s4.c:24-27): "M:" lines (s4.c:250-253), "5:" / 6-set / drill lines
 * through format_set (s4.c:214-220), "4:" dump lines (s4.c:239).
 *
 * Pure formatting: every number and every verify flag comes from the device records.
 */
#include <stdio.h>
#include <string.h>

#include "../../include/ps4.h"

typedef unsigned __int128 u128;

typedef struct { char *p; size_t cap, len; int bad; } sbuf;

static void put(sbuf *b, const char *s, size_t n) {
    if (b->bad || b->len + n + 1 > b->cap) { b->bad = 1; return; }
    memcpy(b->p + b->len, s, n);
    b->len += n;
}
#define PUTS(b, lit) put((b), (lit), sizeof(lit) - 1)

/* decimal digits two at a time from a 200-byte pair table; 128-bit values are cut into
 * 19-digit blocks first (one 128-bit division per block), so the digit loop runs on 64 bits */
static const char DIG2[201] =
    "00010203040506070809101112131415161718192021222324252627282930313233343536373839"
    "40414243444546474849505152535455565758596061626364656667686970717273747576777879"
    "8081828384858687888990919293949596979899";

static int u64_digits(char *end, unsigned long long v) {  /* writes backwards from end, returns count */
    char *p = end;
    while (v >= 100) {
        const unsigned r = (unsigned)(v % 100);
        v /= 100;
        p -= 2;
        memcpy(p, DIG2 + 2 * r, 2);
    }
    if (v >= 10) { p -= 2; memcpy(p, DIG2 + 2 * v, 2); }
    else *--p = (char)('0' + (int)v);
    return (int)(end - p);
}

static void put_u64(sbuf *b, unsigned long long v) {
    char tmp[24];
    const int n = u64_digits(tmp + sizeof tmp, v);
    put(b, tmp + sizeof tmp - n, (size_t)n);
}

static void put_u128(sbuf *b, u128 v) {
    if ((v >> 64) == 0) { put_u64(b, (unsigned long long)v); return; }
    const unsigned long long E19 = 10000000000000000000ull;
    char tmp[48];
    char *end = tmp + sizeof tmp, *p = end;
    while ((v >> 64) != 0) {                   /* low 19-digit blocks, zero-padded */
        const unsigned long long blk = (unsigned long long)(v % E19);
        v /= E19;
        const int n = u64_digits(p, blk);
        p -= n;
        for (int k = n; k < 19; k++) *--p = '0';
    }
    p -= u64_digits(p, (unsigned long long)v);
    put(b, p, (size_t)(end - p));
}

static u128 ext_value(const ps4_ext *e) { return ((u128)e->hi << 64) | e->lo; }

/* "tag [x sorted descending] S=...<verify note>\n" */
static void put_set(sbuf *b, const char *tag, u128 *x, int n, uint64_t S, int verified) {
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
            if (x[j] > x[i]) { u128 t = x[i]; x[i] = x[j]; x[j] = t; }
    put(b, tag, strlen(tag));
    PUTS(b, " [");
    for (int i = 0; i < n; i++) {
        put_u128(b, x[i]);
        if (i < n - 1) put(b, ",", 1);
    }
    PUTS(b, "] S=");
    put_u64(b, S);
    if (!verified) PUTS(b, "  *** VERIFY FAILED ***");
    put(b, "\n", 1);
}

static long done(sbuf *b) {
    if (b->bad) return -1;
    b->p[b->len] = 0;                          /* put() keeps one byte free for it */
    return (long)b->len;
}

long ps4_format_hit(const ps4_hit *h, const ps4_ext *exts, char *buf, size_t cap) {
    sbuf b = {buf, cap, 0, cap == 0};
    if (cap) buf[0] = 0;
    const ps4_ext *e = exts + h->first_ext;
    if (h->n_ext >= 2) {
        PUTS(&b, "M: [");
        for (int i = 0; i < 4; i++) { put_u64(&b, h->v[i]); if (i < 3) put(&b, ",", 1); }
        PUTS(&b, "] ext=[");
        for (uint32_t t = 0; t < h->n_ext; t++) {
            put_u128(&b, ext_value(&e[t]));
            if (t + 1 < h->n_ext) put(&b, ",", 1);
        }
        PUTS(&b, "] S=");
        put_u64(&b, h->S);
        put(&b, "\n", 1);
    }
    for (uint32_t t = 0; t < h->n_ext; t++) {
        if (!(e[t].flags & PS4_EXT_FIVE)) continue;
        u128 x[5] = {h->v[0], h->v[1], h->v[2], h->v[3], ext_value(&e[t])};
        put_set(&b, "5:", x, 5, h->S, (e[t].flags & PS4_EXT_FIVE_OK) != 0);
    }
    return done(&b);
}

long ps4_format_hits(const ps4_hit *hits, uint64_t n, const ps4_ext *exts, char *buf, size_t cap,
                     uint32_t *line_items, uint64_t *n_lines) {
    char tmp[8192];
    size_t len = 0;
    uint64_t lines = 0;
    int full = 0;
    if (cap) buf[0] = 0;
    for (uint64_t i = 0; i < n; i++) {
        char *dst = full ? tmp : buf + len;
        size_t room = full ? sizeof tmp : cap - len;
        long k = ps4_format_hit(&hits[i], exts, dst, room);
        if (k < 0 && !full) {                  /* buf is too small: keep counting the length */
            full = 1;
            if (len < cap) buf[len] = 0;       /* end at the last complete hit */
            k = ps4_format_hit(&hits[i], exts, tmp, sizeof tmp);
            dst = tmp;
        }
        if (k < 0) return -1;                  /* a single hit longer than 8 KB: not produced by a search */
        /* its lines: the M line (two or more extensions) and one 5: line per extension above max(v) */
        const ps4_ext *e = exts + hits[i].first_ext;
        uint32_t nh = hits[i].n_ext >= 2 ? 1u : 0u;
        for (uint32_t t = 0; t < hits[i].n_ext; t++) nh += (e[t].flags & PS4_EXT_FIVE) ? 1u : 0u;
        if (line_items && !full)
            for (uint32_t j = 0; j < nh; j++) line_items[lines + j] = hits[i].item;
        lines += nh;
        len += (size_t)k;
    }
    if (n_lines) *n_lines = lines;
    return full ? -(long)(len + 1) : (long)len;
}

long ps4_format_six(const ps4_hit *h, const ps4_ext *exts, const ps4_six *s, char *buf, size_t cap) {
    sbuf b = {buf, cap, 0, cap == 0};
    if (cap) buf[0] = 0;
    const ps4_ext *e = exts + h->first_ext;
    u128 x[6] = {h->v[0], h->v[1], h->v[2], h->v[3], ext_value(&e[s->t]), ext_value(&e[s->s])};
    put_set(&b, "!!!!!!!! FOUND 6-SET:", x, 6, h->S, (s->flags & 1) != 0);
    return done(&b);
}

long ps4_format_drill(const ps4_hit *h, const ps4_ext *exts, char *buf, size_t cap) {
    sbuf b = {buf, cap, 0, cap == 0};
    if (cap) buf[0] = 0;
    if (h->n_ext < 2) return 0;
    const ps4_ext *e = exts + h->first_ext;
    u128 x[6] = {h->v[0], h->v[1], h->v[2], h->v[3], ext_value(&e[0]), ext_value(&e[1])};
    put_set(&b, "TEST-6SET (NOT A SOLUTION, --test-sixset drill):", x, 6, h->S, (h->flags & PS4_HIT_DRILL_OK) != 0);
    return done(&b);
}

void ps4_quad_values(const ps4_quad *q, uint64_t *S, uint64_t v[4], uint32_t order[4]) {
    uint64_t ab = (uint64_t)q->r_ab * q->r_ab, ac = (uint64_t)q->r_ac * q->r_ac, ad = (uint64_t)q->r_ad * q->r_ad;
    uint64_t bc = (uint64_t)q->r_bc * q->r_bc, cd = (uint64_t)q->r_cd * q->r_cd;
    uint64_t a = (ab + ac - bc) >> 1;
    v[0] = a; v[1] = ab - a; v[2] = ac - a; v[3] = ad - a;
    *S = ab + cd;
    order[0] = q->r_cd;                                   /* p of representation x */
    order[1] = q->r_bd;                                   /* p of representation y */
    order[2] = q->r_ad < q->r_bc ? q->r_ad : q->r_bc;      /* p of representation z */
    order[3] = q->r_ad < q->r_bc ? 1u : 0u;                /* class */
}

long ps4_format_quad(const ps4_quad *q, char *buf, size_t cap) {
    uint64_t S, v[4];
    uint32_t order[4];
    ps4_quad_values(q, &S, v, order);
    int n = snprintf(buf, cap, "4: [%lld,%lld,%lld,%lld] S=%llu\n", (long long)v[0], (long long)v[1], (long long)v[2],
                     (long long)v[3], (unsigned long long)S);
    return (n < 0 || (size_t)n >= cap) ? -1 : n;
}
