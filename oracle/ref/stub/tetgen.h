/* Placeholder for the third-party TetGen header.  The reference only needs
 * the type names to compile Domain.C; the mesh paths that would call TetGen
 * are never reached by the oracle driver. */
#pragma once
class tetgenio { public: };
class tetgenbehavior { public: };
