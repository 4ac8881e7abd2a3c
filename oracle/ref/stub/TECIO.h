/* Placeholder for the third-party Tecplot I/O header.  The binary Tecplot
 * writer of Output3D.C links against these; each stub in ref_stubs.C
 * returns -1 ("failed"), so only the VTK/GNU writers produce output. */
#pragma once
int TECINI112(...);
int TECZNE112(...);
int TECDAT112(...);
int TECNOD112(...);
int TECEND112(...);
int TECEND(...);
