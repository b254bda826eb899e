/* Umbrella header of the gzg system-library module: the C ABI of libgzg.so. */
#include <gzg.h>
