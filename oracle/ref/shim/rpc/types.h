/* Minimal stand-in for <rpc/types.h>: the reference headers (pbf.h) include it when
 * HDF5 is off; no XDR routine is called on the solver path. Test infrastructure only. */
typedef struct { int x_op; } XDR;
typedef int bool_t;
