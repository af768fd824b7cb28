/* Empty stand-in: massive_block_proj.cu includes thrust headers but calls
 * thrust only in comments (host build, oracle/_ref). */
