/*
 * story_oracle.c -- TEST INFRASTRUCTURE (the oracle): Starlab's reader of
 * story-format snapshots for the dyn class, restated sequentially in C.
 *
 * It follows get_dyn -> get_node (src/node/util/tree_io.C:253-410) line by
 * line, with the reference's own rules:
 *   * a line is at most 254 characters, the rest is discarded (get_line,
 *     src/std/util_io.C:22-40); inside a Log story a longer line is an error
 *     (get_story_line, src/std/story.C:61-75);
 *   * section lines are recognised by their first two characters after
 *     skipping every byte that compares <= ' ' as a (signed) char
 *     (matchbracket, util_io.C:94-109): "(P"/")P", "(D"/")D", "(H"/")H",
 *     "(S"/")S", "(L";
 *   * a Dynamics section runs to the first ")D" line (scan_dyn_story,
 *     src/node/dyn/util/dyn_io.C:148-206): "m" (strtod), "r" and "v" (three
 *     strtod, error if the third converts nothing, util_io.C:145-157),
 *     "system_time" (strtod; this build reads xreal as real), other lines
 *     kept as story text (ignored here);
 *   * Hydro and Star sections run to the first ")H" / ")S" line
 *     (hydrobase_io.C:17-27, starbase_io.C:18+); their contents are not dyn
 *     data;
 *   * a Log story is a chapter read by its raw first character, '(' opening
 *     and ')' closing sub-chapters whose closing title must equal the
 *     opening one (get_chapter, story.C:172-203);
 *   * in a particle body: "i" (strtol), "name" (first token), "N"
 *     (ignored), any other "keyword = value" is an error (tree_io.C:323-343);
 *     lines without '=' are ignored;
 *   * snapshots follow one another until an empty line or the end of the
 *     text (check_and_skip_input_line, util_io.C:54-82);
 *   * unless raw, check_and_correct_node (dyn_io.C:94-146) then sets every
 *     parent's mass to the sum of its daughters' (in daughter order, post
 *     order) and moves the daughters to their centre-of-mass frame.
 * Where the reference exits (or reads past its buffer) this returns an
 * error with the line number instead.
 *
 * Output, over all snapshots in document (pre-)order: parent (-1 for a
 * root), index label (-1: none), name (offset and length in the text, -1:
 * none), mass, pos[3], vel[3]; per root its node and the system time the
 * reference's static dyn::system_time holds after reading it.  Leaf
 * positions relative to the root (something_relative_to_root,
 * src/node/dyn/util/dyn_tt.C:94-110) are left to the caller.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <ctype.h>

#define LINE_MAX_CHARS 254

typedef struct {
    const char *t;
    long long len, pos;
    long long line_no;   /* 1-based number of the last line read */
} Src;

typedef struct {
    long long n, cap;
    int *parent, *index, *name_off, *name_len;
    double *mass, *pos, *vel;
    long long nr, rcap;
    int *root_node;
    double *root_time;
    long long err_line;
    int err;
    const char *err_what;
} Tree;

static void grow_nodes(Tree *T)
{
    if (T->n < T->cap) return;
    long long c = T->cap ? 2 * T->cap : 1024;
    T->parent = realloc(T->parent, 4 * c);
    T->index = realloc(T->index, 4 * c);
    T->name_off = realloc(T->name_off, 4 * c);
    T->name_len = realloc(T->name_len, 4 * c);
    T->mass = realloc(T->mass, 8 * c);
    T->pos = realloc(T->pos, 24 * c);
    T->vel = realloc(T->vel, 24 * c);
    T->cap = c;
}

/* Next line: *b = its start, returns its length after truncation; -1 at
 * the end of the text.  *full = untruncated length. */
static int next_line(Src *s, const char **b, long long *full)
{
    if (s->pos >= s->len) return -1;
    const char *p = s->t + s->pos;
    const char *nl = memchr(p, '\n', (size_t)(s->len - s->pos));
    long long L = nl ? (long long)(nl - p) : s->len - s->pos;
    s->pos += L + (nl ? 1 : 0);
    s->line_no++;
    *b = p;
    *full = L;
    return (int)(L > LINE_MAX_CHARS ? LINE_MAX_CHARS : L);
}

static int fail(Tree *T, Src *s, const char *what)
{
    if (!T->err) {
        T->err = 1;
        T->err_line = s->line_no;
        T->err_what = what;
    }
    return -1;
}

/* matchbracket over a line of n characters: the first two characters after
 * the skipped ones, a character past the end never matching. */
static int match2(const char *l, int n, char a, char b)
{
    int k = 0;
    while (k < n && (signed char)l[k] <= ' ') ++k;
    return k + 1 < n && l[k] == a && l[k + 1] == b;
}

/* getequals: keyword into kw (NUL-terminated), returns the value offset or
 * -1 without '='. */
static int getequals(const char *l, int n, char *kw)
{
    int k = 0, i = 0;
    while (k < n && isspace((unsigned char)l[k])) ++k;
    while (k < n && (isalnum((unsigned char)l[k]) || l[k] == '_') && !((unsigned char)l[k] & 0x80)) kw[i++] = l[k++];
    kw[i] = 0;
    while (k < n && l[k] != '=') ++k;
    if (k >= n) return -1;
    ++k;
    while (k < n && isspace((unsigned char)l[k])) ++k;
    return k;
}

/* strtod / strtol on a line's value, the line ending at n characters. */
static double line_strtod(const char *l, int n, int off, int *used)
{
    char buf[LINE_MAX_CHARS + 1];
    memcpy(buf, l, (size_t)n);
    buf[n] = 0;
    char *end;
    double v = strtod(buf + off, &end);
    *used = (int)(end - (buf + off));
    return v;
}

static long line_strtol(const char *l, int n, int off)
{
    char buf[LINE_MAX_CHARS + 1];
    memcpy(buf, l, (size_t)n);
    buf[n] = 0;
    return strtol(buf + off, NULL, 10);
}

static int read_vector(const char *l, int n, double *v)
{
    const char *eq = memchr(l, '=', (size_t)n);
    int off = (int)(eq - l) + 1, u0, u1, u2;
    v[0] = line_strtod(l, n, off, &u0);
    off += u0;
    v[1] = line_strtod(l, n, off, &u1);
    off += u1;
    v[2] = line_strtod(l, n, off, &u2);
    return u2 > 0 ? 0 : -1;
}

static double g_system_time = 0.0; /* the reference's static dyn::system_time */

static int scan_dyn(Tree *T, Src *s, long long node)
{
    const char *l;
    long long full;
    int n;
    char kw[LINE_MAX_CHARS + 1];
    for (;;) {
        if ((n = next_line(s, &l, &full)) < 0) return fail(T, s, "end of text inside Dynamics");
        if (match2(l, n, ')', 'D')) return 0;
        int off = getequals(l, n, kw);
        if (off < 0) continue;
        int used;
        if (!strcmp(kw, "real_system_time")) {
            /* only selects the xreal reading of system_time (read as real here) */
        } else if (!strcmp(kw, "system_time")) {
            g_system_time = line_strtod(l, n, off, &used);
        } else if (!strcmp(kw, "m")) {
            T->mass[node] = line_strtod(l, n, off, &used);
        } else if (!strcmp(kw, "r")) {
            if (read_vector(l, n, T->pos + 3 * node)) return fail(T, s, "expected three reals");
        } else if (!strcmp(kw, "v")) {
            if (read_vector(l, n, T->vel + 3 * node)) return fail(T, s, "expected three reals");
        }
    }
}

static int skip_to(Tree *T, Src *s, char kind)
{
    const char *l;
    long long full;
    int n;
    for (;;) {
        if ((n = next_line(s, &l, &full)) < 0) return fail(T, s, "end of text inside a section");
        if (match2(l, n, ')', kind)) return 0;
    }
}

static int chapter(Tree *T, Src *s, const char *open, int on)
{
    if (open[0] != '(') return fail(T, s, "chapter line does not begin with '('");
    const char *l;
    long long full;
    int n;
    for (;;) {
        if ((n = next_line(s, &l, &full)) < 0) return fail(T, s, "end of text inside a story chapter");
        if (full > LINE_MAX_CHARS) return fail(T, s, "story line too long");
        if (n == 0) return fail(T, s, "empty line inside a story chapter");
        if (l[0] == ')') {
            if (n != on || memcmp(l + 1, open + 1, (size_t)(n - 1))) return fail(T, s, "chapter closing title differs");
            return 0;
        }
        if (l[0] == '(' && chapter(T, s, l, n)) return -1;
    }
}

static long long particle(Tree *T, Src *s, long long parent)
{
    grow_nodes(T);
    const long long me = T->n++;
    T->parent[me] = (int)parent;
    T->index[me] = -1;
    T->name_off[me] = -1;
    T->name_len[me] = 0;
    T->mass[me] = 1.0;
    for (int c = 0; c < 3; ++c) T->pos[3 * me + c] = T->vel[3 * me + c] = 0.0;
    const char *l;
    long long full;
    int n;
    char kw[LINE_MAX_CHARS + 1];
    for (;;) {
        if ((n = next_line(s, &l, &full)) < 0) return fail(T, s, "end of text inside a Particle");
        if (match2(l, n, ')', 'P')) return me;
        if (match2(l, n, '(', 'D')) {
            if (scan_dyn(T, s, me)) return -1;
        } else if (match2(l, n, '(', 'H')) {
            if (skip_to(T, s, 'H')) return -1;
        } else if (match2(l, n, '(', 'S')) {
            if (skip_to(T, s, 'S')) return -1;
        } else if (match2(l, n, '(', 'L')) {
            if (chapter(T, s, l, n)) return -1;  /* title: the line as get_line kept it */
        } else if (match2(l, n, '(', 'P')) {
            if (particle(T, s, me) < 0) return -1;
        } else {
            int off = getequals(l, n, kw);
            if (off < 0) continue;
            if (!strcmp(kw, "i")) {
                T->index[me] = (int)line_strtol(l, n, off);
            } else if (!strcmp(kw, "name")) {
                int k = off;
                while (k < n && !isspace((unsigned char)l[k])) ++k;
                T->name_off[me] = (int)((l + off) - s->t);
                T->name_len[me] = k - off;
            } else if (!strcmp(kw, "N")) {
            } else {
                return fail(T, s, "unexpected keyword in a Particle");
            }
        }
    }
}

/* check_and_correct_node, post order, daughters in order. */
static void correct(Tree *T, long long b, long long end)
{
    /* daughters of b: the nodes in (b, end) whose parent is b */
    double m = 0, p[3] = {0, 0, 0}, v[3] = {0, 0, 0};
    int has = 0;
    long long d = b + 1;
    while (d < end) {
        long long e = d + 1;
        while (e < end && T->parent[e] != (int)b) ++e;  /* d's subtree is [d, e) */
        if (e > d + 1) correct(T, d, e);
        double mm = T->mass[d];
        m += mm;
        for (int c = 0; c < 3; ++c) {
            p[c] += mm * T->pos[3 * d + c];
            v[c] += mm * T->vel[3 * d + c];
        }
        has = 1;
        d = e;
    }
    if (!has) return;
    T->mass[b] = m;
    if (m > 0) {
        for (int c = 0; c < 3; ++c) {
            p[c] /= m;
            v[c] /= m;
        }
        for (d = b + 1; d < end; ++d)
            if (T->parent[d] == (int)b)
                for (int c = 0; c < 3; ++c) {
                    T->pos[3 * d + c] += -p[c];
                    T->vel[3 * d + c] += -v[c];
                }
    }
}

void *so_parse(const char *text, long long len, int raw, long long *n_nodes, long long *n_roots, long long *err_line,
               const char **err_what)
{
    Tree *T = calloc(1, sizeof(Tree));
    Src s = {text, len, 0, 0};
    g_system_time = 0.0;
    if (memchr(text, 0, (size_t)len)) {
        T->err = 1;
        T->err_what = "NUL byte in the text";
    }
    while (!T->err) {
        const char *l;
        long long full;
        int n = next_line(&s, &l, &full);
        if (n <= 0) break; /* end of text, or an empty line: no more snapshots */
        if (!match2(l, n, '(', 'P')) {
            if (s.pos >= s.len && text[len - 1] != '\n') break; /* an unterminated last line ends the input */
            fail(T, &s, "expected (Particle");
            break;
        }
        long long r = particle(T, &s, -1);
        if (r < 0) break;
        if (!raw && T->n - r > 1) correct(T, r, T->n);
        if (T->nr == T->rcap) {
            T->rcap = T->rcap ? 2 * T->rcap : 16;
            T->root_node = realloc(T->root_node, 4 * T->rcap);
            T->root_time = realloc(T->root_time, 8 * T->rcap);
        }
        T->root_node[T->nr] = (int)r;
        T->root_time[T->nr] = g_system_time;
        T->nr++;
    }
    *n_nodes = T->n;
    *n_roots = T->nr;
    *err_line = T->err ? T->err_line : 0;
    *err_what = T->err ? T->err_what : NULL;
    return T;
}

int so_error(void *h) { return ((Tree *)h)->err; }

void so_get(void *h, int *parent, int *index, int *name_off, int *name_len, double *mass, double *pos, double *vel,
            int *root_node, double *root_time)
{
    Tree *T = h;
    const size_t n = (size_t)T->n, r = (size_t)T->nr;
    if (parent) memcpy(parent, T->parent, 4 * n);
    if (index) memcpy(index, T->index, 4 * n);
    if (name_off) memcpy(name_off, T->name_off, 4 * n);
    if (name_len) memcpy(name_len, T->name_len, 4 * n);
    if (mass) memcpy(mass, T->mass, 8 * n);
    if (pos) memcpy(pos, T->pos, 24 * n);
    if (vel) memcpy(vel, T->vel, 24 * n);
    if (root_node) memcpy(root_node, T->root_node, 4 * r);
    if (root_time) memcpy(root_time, T->root_time, 8 * r);
}

void so_free(void *h)
{
    Tree *T = h;
    if (!T) return;
    free(T->parent); free(T->index); free(T->name_off); free(T->name_len);
    free(T->mass); free(T->pos); free(T->vel); free(T->root_node); free(T->root_time);
    free(T);
}
