// szsnn_locales.h -- layout constants for building the reference's host with
// the szsnn compat layer.  Force-included ahead of every reference source
// (-include), it defines the include guard of the reference's locales.h, so
// that file's body (whose active values are a 32-neuron debugging layout)
// is skipped and the macros below take its place.  The names are the
// reference's (locales.h:18-70): the host and the drop-in kernels must agree
// on them.  Values: the production layout the reference keeps beside its
// debugging one (MAX_PARTITION_SIZE 1024, WARP_SIZE 32, NEURONS_PER_WI 4,
// MAX_SYNAPTIC_DELAY 64), or a smaller partition with -DSZSNN_MPS=256.
#ifndef LOCALES_H_
#define LOCALES_H_

#ifndef SZSNN_MPS
#define SZSNN_MPS 1024
#endif

#define MAX_CONNECTIONS_PER_NEURON (1 << 10)
#define MAX_PARTITION_SIZE SZSNN_MPS
#define MAX_PARTITION_COUNT (1 << 10)
#define MAX_INPUTS_SIZE MAX_PARTITION_SIZE
#define MAX_NETWORK_SIZE MAX_PARTITION_COUNT * MAX_PARTITION_SIZE
#define BIT_VECTOR_WORD_SIZE 32
#define BIT_VECTOR_BYTE_PITCH ((MAX_PARTITION_SIZE) / 8)
#define BIT_VECTOR_WORD_PITCH ((MAX_PARTITION_SIZE) / (BIT_VECTOR_WORD_SIZE))
#define WARP_SIZE 32
#define BUNDLE_SIZE WARP_SIZE
#define NEURONS_PER_WI 4
#define THREADS_PER_GROUP ((MAX_PARTITION_SIZE) / (NEURONS_PER_WI))
#define WARPS_PER_GROUP (THREADS_PER_GROUP / WARP_SIZE)
#define MIN_SYNAPTIC_DELAY 1
#define MAX_SYNAPTIC_DELAY 64
#define SZSNN_COMMENT_CHAR '#'
#define SZSNN_ROOT_PATH ""
#define SZSNN_SRC_PATH ""
#define SZSNN_SRC_CL_PATH ""
#define SZSNN_CONFIG_PATH ""
#define TARGET_DEVICE_NAME "szsnn sm_100a"
#define OCL_COMPILER_OPTIONS_FILE_NAME ""
#define _SZSNN_NONE_KERNEL "__NONE"
#define SZSNN_NO_INPUT_TO_OUTPUT 1

#endif
