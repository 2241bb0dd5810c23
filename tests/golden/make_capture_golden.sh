#!/bin/sh
# Writes the capture fixtures with the reference's own header-only writers
# (compiled by oracle/Makefile into oracle/_ref/capture_writer from
# fast_rap_src_dfpt_gpu_eval/*_direct_test.hpp); run from the repository root
# after `make -C oracle`.
set -e
oracle/_ref/capture_writer tests/golden/capture_rho_meta.bin tests/golden/capture_sumup.bin
