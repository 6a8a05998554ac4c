/*
 * Host-side harness around the reference's own deletion-variant generator and codec.
 *
 * TEST INFRASTRUCTURE ONLY. build_ref.sh compiles this file against the reference sources
 * where they lie (include path given on the command line) into oracle/_ref/ref_harness.
 * With TEST_ENV defined the reference marks expand_keys() __host__
 * (S/src/generate_combination.cu:35-41), so it runs without a GPU. The tests feed it random
 * sequences and compare its output with the CPU restatement in oracle.cpp.
 *
 * stdin : one "SEQUENCE DISTANCE" per line
 * stdout: "E w0 w1 w2 len" for str_encode/len_decode, then "R pos w0 w1 w2" per position for
 *         remove_char, then "V count" followed by one line per variant "w0 w1 w2".
 */
#include <stdio.h>
#include <string.h>
#include <vector>
#include <string>
#define TEST_ENV
#include "generate_combination.cu"

int main() {
	char seq[64];
	int d;
	while (scanf("%63s %d", seq, &d) == 2) {
		Int3 v = str_encode(seq);
		int len = len_decode(v);
		printf("E %u %u %u %d\n", v.entry[0], v.entry[1], v.entry[2], len);
		for (int p = 0; p < len; p++) {
			Int3 r = remove_char(v, p);
			printf("R %d %u %u %u\n", p, r.entry[0], r.entry[1], r.entry[2]);
		}
		int e = d < len ? d : len;
		long total = 0, c = 1;
		for (int k = 0; k <= e; k++) {
			total += c;
			c = c * (len - k) / (k + 1);
		}
		Int3* out = new Int3[total];
		unsigned int* fk = new unsigned int[total];
		expand_keys(v, d, out, fk, 0, (int)total);
		printf("V %ld\n", total);
		for (long i = 0; i < total; i++)
			printf("%u %u %u\n", out[i].entry[0], out[i].entry[1], out[i].entry[2]);
		delete[] out;
		delete[] fk;
	}
	return 0;
}
