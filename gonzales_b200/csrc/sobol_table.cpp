// sobol_table.cpp - embeds gonzales_b200/data/sobol_1024x52.bin (the Sobol
// generator matrices of Sources/SobolGenerator/main.swift, 1024 dimensions x 52
// uint32 columns, little-endian, dimension-major) into libgzg.so.
#include <cstddef>
#include <cstdint>

#ifndef GZG_SOBOL_PATH
#error "GZG_SOBOL_PATH must name sobol_1024x52.bin"
#endif

#define GZG_STR2(x) #x
#define GZG_STR(x) GZG_STR2(x)

asm(".section .rodata\n"
    ".balign 64\n"
    ".global gzg_sobol_blob\n"
    ".hidden gzg_sobol_blob\n"
    "gzg_sobol_blob:\n"
    ".incbin \"" GZG_STR(GZG_SOBOL_PATH) "\"\n"
    ".global gzg_sobol_blob_end\n"
    ".hidden gzg_sobol_blob_end\n"
    "gzg_sobol_blob_end:\n"
    ".previous\n");

extern "C" const unsigned char gzg_sobol_blob[];
extern "C" const unsigned char gzg_sobol_blob_end[];

namespace gzg {

const uint32_t *sobol_matrices(size_t *count) {
        *count = (size_t)(gzg_sobol_blob_end - gzg_sobol_blob) / sizeof(uint32_t);
        return reinterpret_cast<const uint32_t *>(gzg_sobol_blob);
}

}  // namespace gzg
