/* Embeds the MT19937 jump polynomials (made at build time by
   rocrand_b200/data/make_mt19937_jump.c) into liborc.so (test infrastructure only). */
    .section .note.GNU-stack,"",@progbits
    .section .rodata
    .globl orc_mt19937_jump_begin
    .p2align 4
orc_mt19937_jump_begin:
    .incbin "mt19937_jump.bin"
