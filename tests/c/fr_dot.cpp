// Host build of the BN254 scalar-field arithmetic (zeknox_b200/csrc/bn254.cuh,
// the code the device compiles too): for each input line of ten field
// elements a0 b0 .. a4 b4 (64 hex digits each, canonical, plain form) it
// prints the five-term dot product sum a_j * b_j * 2^-256 mod r twice, as one
// reduction of the 512-bit sum (fr_mac_wide, fr_reduce_wide) and as five
// Montgomery products added one by one (fr_mul, fr_add).
#include <stdio.h>
#include <string.h>

#include "bn254.cuh"

using zk::Fr;

static bool parse(const char *h, Fr &x)
{
    if (strlen(h) != 64) return false;
    for (int i = 0; i < 8; i++) {
        unsigned v = 0;
        if (sscanf(h + 8 * (7 - i), "%8x", &v) != 1) return false;
        x.w[i] = v;
    }
    return true;
}

static void print(const Fr &x)
{
    for (int i = 7; i >= 0; i--) printf("%08x", x.w[i]);
}

int main()
{
    char tok[10][80];
    while (scanf("%79s %79s %79s %79s %79s %79s %79s %79s %79s %79s", tok[0], tok[1], tok[2], tok[3], tok[4], tok[5],
                 tok[6], tok[7], tok[8], tok[9]) == 10) {
        Fr a[5], b[5];
        for (int j = 0; j < 5; j++)
            if (!parse(tok[2 * j], a[j]) || !parse(tok[2 * j + 1], b[j])) return 2;
        zk::FrWide acc;
        zk::fr_wide_zero(acc);
        for (int j = 0; j < 5; j++) acc = zk::fr_mac_wide_ol(acc, a[j], b[j]);
        const Fr one = zk::fr_reduce_wide_ol(acc);
        Fr five = zk::fr_mul(a[0], b[0]);
        for (int j = 1; j < 5; j++) five = zk::fr_add(five, zk::fr_mul(a[j], b[j]));
        print(one);
        printf(" ");
        print(five);
        printf("\n");
    }
    return 0;
}
