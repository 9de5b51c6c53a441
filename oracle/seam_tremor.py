"""Writes the reference's Tremor.cpp with the GPU worker seam (test infrastructure).

    python oracle/seam_tremor.py <reference Tremor.cpp> <output Tremor.cpp>

The output is the reference's own file with two edits a maintainer would make to route the
adaptive planner's scan and FFT branches to the GPU (include/tremor_b200_worker_seam.hpp):
the seam header is included just before the definition of refine_in_position_order, and
the two branch calls of the planner's worker (Tremor.cpp:2293-2296) call
tm_gpu_in_position_order instead. Each edit must apply exactly once, else nothing is
written. The output goes under oracle/_ref/ (not committed); the reference's relative
includes resolve through -iquote of its directory (oracle/Makefile, target driver-gpu)."""
import sys

CALLS = ('fft_in_position_order(in_data);', 'refine_in_position_order(in_data, bounds_prune);')
DEFINITION = 'static void refine_in_position_order(QaWorkerData *in_data, bool use_lb)'


def main(src, dst):
    text = open(src).read()
    for call in CALLS:
        hits = [i for i, line in enumerate(text.splitlines()) if line.strip() == call]
        if len(hits) != 1:
            sys.exit(f'seam_tremor: expected one line "{call}", found {len(hits)}')
        text = text.replace(call, 'tm_gpu_in_position_order(in_data);', 1)
    if text.count(DEFINITION) != 1:
        sys.exit('seam_tremor: definition of refine_in_position_order not found once')
    text = text.replace(DEFINITION, '#include "tremor_b200_worker_seam.hpp"\n\n' + DEFINITION, 1)
    with open(dst, 'w') as f:
        f.write(text)


if __name__ == '__main__':
    main(sys.argv[1], sys.argv[2])
