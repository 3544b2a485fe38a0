/* gpujoind wire protocol, byte-compatible with landstats-us/postgis-cuda daemon/protocol.h:1-44, so the
 * gpu_spatial Postgres extension (ext/gpu_spatial.c) talks to gsjd unchanged. Little endian throughout.
 *
 * request : u32 GSP_MAGIC, u32 op, u32 nargs (<= 64), nargs x { u32 len (<= 64 MiB), bytes }
 *           args[0] is the auth token (empty when the daemon runs without a token); the op's args follow.
 * response: u32 status (GSP_OK / GSP_ERR); GSP_ERR is followed by u32 len, message.
 *   JSON ops (LOAD, LOAD_QUERY, DROP, STATUS, LIST): u32 len, JSON text.
 *   stream ops (JOIN, CLUSTER, RELATE, DWITHIN): frames { u32 nrows, rows } of at most ~1 MiB, ended by
 *   nrows == 0 followed by u32 len, JSON stats; nrows == GSP_FRAME_ERR is followed by u32 len, message.
 *   join / dwithin row : u16 la, a_id[la], u16 lb, b_id[lb], f64 area (NaN without area; always NaN for DWITHIN)
 *   cluster row        : u16 l, id[l], u32 cluster
 *   relate row         : u16 la, a_id[la], u16 lb, b_id[lb], char[9] DE-9IM matrix
 *
 * op args (UTF-8 strings):
 *   LOAD       layer, table, id_col, geom_col, filter, subdivide, dedup
 *   LOAD_QUERY layer, sql, subdivide, dedup
 *   DROP       layer
 *   LIST / STATUS
 *   JOIN       layer_a, layer_b, want_area ("1"/"0"), self_pairs ("all" | "distinct")[, "stats"]
 *   CLUSTER    layer
 *   RELATE     layer_a, layer_b, pattern ("" = every intersecting pair), self_pairs
 *   DWITHIN    layer_a, layer_b, mode ("dwithin" | "buffer"), dist_a, dist_b, self_pairs[, "stats"]   (meters)
 */
#ifndef GSP_PROTOCOL_H
#define GSP_PROTOCOL_H

#define GSP_MAGIC 0x52505347u /* "GSPR" read as a little-endian u32 */
#define GSP_OK 0u
#define GSP_ERR 1u
#define GSP_FRAME_ERR 0xFFFFFFFFu
#define GSP_MAX_ARGS 64u
#define GSP_MAX_ARG_BYTES (64u << 20)
#define GSP_FRAME_BYTES (1u << 20) /* a frame is closed once it holds this many bytes of rows */

enum gsp_op {
  GSP_OP_LOAD = 1,
  GSP_OP_LOAD_QUERY = 2,
  GSP_OP_DROP = 3,
  GSP_OP_LIST = 4,
  GSP_OP_STATUS = 5,
  GSP_OP_JOIN = 6,
  GSP_OP_CLUSTER = 7,
  GSP_OP_RELATE = 8,
  GSP_OP_DWITHIN = 9
};

#endif
