#!/bin/bash
# The CPU features a g++ target (-march=$1) lets the compiler use, as the
# /proc/cpuinfo flag names a host must show to run code built for it.
# Used to stamp oracle/_ref/athena_ref_native.isa.
set -euo pipefail
march="${1:-native}"
declare -A NAME=([sse3]=pni [bmi]=bmi1 [lzcnt]=abm [sha]=sha_ni [rdrnd]=rdrand
                 [sahf]=lahf_lm [avx512vbmi2]=avx512_vbmi2 [avx512vnni]=avx512_vnni
                 [avx512bitalg]=avx512_bitalg [avx512vpopcntdq]=avx512_vpopcntdq
                 [avx512bf16]=avx512_bf16 [avx512fp16]=avx512_fp16 [avxvnni]=avx_vnni
                 [pclmul]=pclmulqdq [vpclmulqdq]=vpclmulqdq [amx-tile]=amx_tile
                 [amx-int8]=amx_int8 [amx-bf16]=amx_bf16 [sse4.1]=sse4_1 [sse4.2]=sse4_2
                 [cx16]=cx16 [movbe]=movbe [popcnt]=popcnt [f16c]=f16c [fma]=fma
                 [adx]=adx [aes]=aes [gfni]=gfni [vaes]=vaes [rdseed]=rdseed [clwb]=clwb
                 [clflushopt]=clflushopt [avx]=avx [avx2]=avx2 [avx512f]=avx512f
                 [avx512dq]=avx512dq [avx512cd]=avx512cd [avx512bw]=avx512bw
                 [avx512vl]=avx512vl [avx512ifma]=avx512ifma [avx512vbmi]=avx512vbmi
                 [sse]=sse [sse2]=sse2 [ssse3]=ssse3 [bmi2]=bmi2 [xsave]=xsave)
g++ -march="$march" -Q --help=target 2>/dev/null |
  awk '$2 == "[enabled]" && $1 ~ /^-m/ {sub(/^-m/, "", $1); print $1}' |
  while read -r f; do
    if [ -n "${NAME[$f]+x}" ]; then echo "${NAME[$f]}"; fi
  done | sort -u
