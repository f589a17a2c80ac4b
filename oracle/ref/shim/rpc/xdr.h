/* Empty stand-in for <rpc/xdr.h> (see types.h beside it). */
