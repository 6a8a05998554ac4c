/*
 * Timing harness around the reference's own library entry point
 *     void xtn_perform(XTNArgs, SeqArray*, SeqInfo*, void callback(XTNOutput))
 * (xtneighbor_streaming/src/xtn.cu:267), for the reference arm of the benchmark.
 *
 * BENCHMARK INFRASTRUCTURE ONLY, like the other files in this directory. build_ref.sh
 * compiles it against the reference sources where they lie (include path given on the
 * command line) into oracle/_ref/ref_perform. The reference's CLI translation unit
 * (S/src/cli.cu, which includes xtn.cu and airr.cu) is included whole with its main()
 * renamed, so the input parser, the output handler and the search are the reference's own,
 * unmodified code; this file only adds a main() that times repeated searches in one
 * process, so that the reference is measured as a library call, like the build it is
 * compared with (xtn_context_perform), and not as a whole process.
 *
 * usage: ref_perform WARM_CSV WARM_N MAIN_CSV MAIN_N DISTANCE MEASURE STEPS [MAX_SECONDS]
 *   WARM_CSV/WARM_N: a small input in the CLI's format, searched once first (CUDA context
 *                    creation, module loading and first allocations happen there);
 *   MAIN_CSV/MAIN_N: the workload; searched up to STEPS times, stopping early once the timed
 *                    calls have taken MAX_SECONDS in total (at least one call always runs);
 *   MEASURE: 0 Levenshtein, 1 Hamming.
 * Both files are parsed (the reference's parse_input) and moved to the device
 * (SeqArray::toDevice) before any call. Each call is timed by the host clock with a device
 * synchronisation on both sides and the reference's null_handler as the callback, as the
 * CLI does without -o.
 * stdout: "parse <seconds>", "warmup <seconds> <outputs>", then "step <seconds> <outputs>"
 * per timed call, where <outputs> is the number of output entries the callback received.
 */
#include <chrono>

#define main xtn_reference_cli_main
#include "cli.cu"
#undef main

static double seconds_since(std::chrono::steady_clock::time_point t0) {
	return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

static double timed_search(XTNArgs args, SeqArray* seqs, size_t* outputs) {
	cudaDeviceSynchronize();
	totalOutputLen = 0;
	const auto t0 = std::chrono::steady_clock::now();
	xtn_perform(args, seqs, NULL, null_handler);
	cudaDeviceSynchronize();
	const double dt = seconds_since(t0);
	*outputs = totalOutputLen;
	return dt;
}

int main(int argc, char** argv) {
	if (argc < 8) {
		fprintf(stderr, "usage: %s WARM_CSV WARM_N MAIN_CSV MAIN_N DISTANCE MEASURE STEPS [MAX_SECONDS]\n", argv[0]);
		return 1;
	}
	setlocale(LC_ALL, "");
	const int warm_n = atoi(argv[2]), main_n = atoi(argv[4]), steps = atoi(argv[7]);
	const double max_seconds = argc > 8 ? atof(argv[8]) : 1e30;
	XTNArgs warm_args, main_args;
	warm_args.distance = main_args.distance = atoi(argv[5]);
	warm_args.measure = main_args.measure = atoi(argv[6]) ? HAMMING : LEVENSHTEIN;
	warm_args.seqLen = warm_n;
	main_args.seqLen = main_n;
	if (warm_n < 1 || main_n < 1 || warm_args.distance < 1 || steps < 1) {
		fprintf(stderr, "invalid arguments\n");
		return 1;
	}

	SeqArray* warm = new SeqArray(warm_n);
	SeqArray* work = new SeqArray(main_n);
	const auto t0 = std::chrono::steady_clock::now();
	if (parse_input(argv[1], warm, NULL, warm_n, false) != SUCCESS ||
	    parse_input(argv[3], work, NULL, main_n, false) != SUCCESS)
		return 1;
	printf("parse %.6f\n", seconds_since(t0));
	warm->toDevice();
	work->toDevice();

	size_t outputs = 0;
	double dt = timed_search(warm_args, warm, &outputs);
	printf("warmup %.6f %zu\n", dt, outputs);
	fflush(stdout);
	double spent = 0;
	for (int i = 0; i < steps; i++) {
		dt = timed_search(main_args, work, &outputs);
		printf("step %.6f %zu\n", dt, outputs);
		fflush(stdout);
		spent += dt;
		if (spent >= max_seconds)
			break;
	}
	warm->destroy();
	work->destroy();
	return 0;
}
