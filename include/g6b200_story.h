/* g6b200_story.h -- Starlab story-format snapshots read on the GPU.
 *
 * Replaces the dyn-class snapshot reader of the reference, get_dyn(istream&)
 * (src/node/dyn/util/dyn_io.C:280-296, over get_node,
 * src/node/util/tree_io.C:253-410), for large N: the text is parsed on the
 * device and the tree comes back as flat arrays instead of linked dyn nodes.
 * Same results as the reference reader, bit for bit:
 *   - snapshots one after another until an empty line or the end of the text
 *     (check_and_skip_input_line, src/std/util_io.C:54-82);
 *   - per Particle node, in document (pre-)order: its parent (-1 for a
 *     snapshot root), index label "i" (strtol; -1 when absent), name, mass
 *     "m" (strtod; 1 when absent), position "r" and velocity "v" (three
 *     strtod each; 0 when absent) from its Dynamics section, the last line
 *     of a kind winning;
 *   - unless G6B200_STORY_RAW, check_and_correct_node (dyn_io.C:94-146):
 *     every parent's mass becomes the sum of its daughters' and the
 *     daughters are moved to their centre-of-mass frame, with the
 *     reference's order of summation;
 *   - leaves with positions and velocities relative to their root
 *     (something_relative_to_root, src/node/dyn/util/dyn_tt.C:94-110);
 *   - per root, the system time the reference's static dyn::system_time
 *     holds after reading it (the last "system_time" line so far).
 * Where the reference exits or its reading is undefined, or where a form is
 * one this reader does not convert (hexadecimal floats, NaN payloads, more
 * than 40 significant digits, section lines indented by blanks, chapters
 * inside a Dynamics/Hydro/Star section named with that section's letter),
 * parse returns -2 and g6b200_story_error names the line.  Texts of any
 * size below 2^31 - 2 lines (byte offsets are 64-bit). */
#ifndef G6B200_STORY_H
#define G6B200_STORY_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct g6b200_story g6b200_story;

typedef struct {
    long long bytes;    /* bytes of the text read (up to the end of the last snapshot) */
    long long lines;    /* lines read */
    long long n_nodes;  /* Particle nodes of all snapshots */
    long long n_leaves; /* nodes without daughters, roots excluded */
    long long n_roots;  /* snapshots */
    int max_depth;      /* deepest section nesting */
} g6b200_story_info;

#define G6B200_STORY_RAW 1 /* keep the values as written: no check_and_correct_node */

/* A reader with its own CUDA stream and device buffers on `device`, reused
 * from one parse to the next: use a reader from one host thread at a time
 * (one reader per thread for concurrent parses). */
g6b200_story *g6b200_story_create(int device);
void g6b200_story_destroy(g6b200_story *h);
const char *g6b200_story_error(g6b200_story *h);

/* Parse len bytes of story text from host memory (copied to the device), or
 * already on the device (16-byte aligned; only [0, len) is read).  0, -1 on
 * bad arguments or a CUDA error, -2 on a parse error. */
int g6b200_story_parse(g6b200_story *h, const char *text, long long len, int flags, g6b200_story_info *info);
int g6b200_story_parse_device(g6b200_story *h, const char *d_text, long long len, int flags,
                              g6b200_story_info *info);

/* Results of the last successful parse, copied to host arrays (any may be
 * NULL).  Nodes: n_nodes entries.  Names: offset of the name in the text
 * (-1: none) and its length.  Leaves: n_leaves entries, each with its node,
 * index label, mass, and position/velocity relative to its root.  Roots:
 * n_roots entries. */
int g6b200_story_nodes(g6b200_story *h, int *parent, int *index, double *mass, double (*pos)[3],
                       double (*vel)[3]);
int g6b200_story_names(g6b200_story *h, long long *name_offset, int *name_length);
int g6b200_story_leaves(g6b200_story *h, int *node, int *index, double *mass, double (*pos)[3],
                        double (*vel)[3]);
int g6b200_story_roots(g6b200_story *h, int *root_node, double *system_time);
/* Device arrays of the leaves (n_leaves; pos/vel as [n][3]), valid until the
 * next parse or destroy: the j-particles of a force engine, without a copy. */
int g6b200_story_device_leaves(g6b200_story *h, const double **mass, const double **pos, const double **vel);

#ifdef __cplusplus
}
#endif
#endif
