/* Embeds the MT19937 jump polynomials (derived at build time by
   rocrand_b200/data/make_mt19937_jump.c) into librocrand.so. */
    .section .note.GNU-stack,"",@progbits
    .section .rodata
    .globl rb200_mt19937_jump_begin
    .globl rb200_mt19937_jump_end
    .hidden rb200_mt19937_jump_begin
    .hidden rb200_mt19937_jump_end
    .p2align 4
rb200_mt19937_jump_begin:
    .incbin "mt19937_jump.bin"
rb200_mt19937_jump_end:
