/* Embeds rocrand_b200/data/mtgp32_params.bin (the published MTGP32 parameter sets, see
   make_mtgp32_params.py) into librocrand.so. */
    .section .note.GNU-stack,"",@progbits
    .section .rodata
    .globl rb200_mtgp32_params_begin
    .globl rb200_mtgp32_params_end
    .hidden rb200_mtgp32_params_begin
    .hidden rb200_mtgp32_params_end
    .p2align 4
rb200_mtgp32_params_begin:
    .incbin "mtgp32_params.bin"
rb200_mtgp32_params_end:
