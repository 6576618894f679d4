/* Host build of the header-only helpers for CPU unit tests (tests load this
 * through ctypes; the device library compiles the same headers). */
#include "vsg_fpchain.h"

float vsg_test_chain_advance(float r, float h, float target, int max_steps, int* steps) {
    *steps = 0;
    return vsg_chain_advance(r, h, target, max_steps, steps);
}

/* reference: serial additions */
float vsg_test_chain_serial(float r, float h, float target, int max_steps, int* steps) {
    int n = 0;
    while (r < target && n < max_steps) {
        r = r + h;
        ++n;
    }
    *steps = n;
    return r;
}

#include "vsg_mc_table.h"

/* the marching-cubes table the kernel uses, 256 x 16 bytes */
void vsg_test_mc_table(unsigned char* out) { vsg_mc_build_table((unsigned char(*)[16])out); }

/* every case generated by the table's geometric rule, 256 x 16 bytes */
void vsg_test_mc_generated(unsigned char* out) { vsg_mc_generate_table((unsigned char(*)[16])out); }
