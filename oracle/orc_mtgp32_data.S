/* Embeds rocrand_b200/data/mtgp32_params.bin (the published MTGP32 parameter sets) into
   liborc.so (test infrastructure only). */
    .section .note.GNU-stack,"",@progbits
    .section .rodata
    .globl orc_mtgp32_params_begin
    .p2align 4
orc_mtgp32_params_begin:
    .incbin "mtgp32_params.bin"
