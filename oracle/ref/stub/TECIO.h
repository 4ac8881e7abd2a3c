/* Placeholder for the third-party Tecplot I/O header (never called). */
#pragma once
