"""The oracle: test infrastructure that checks the product (never imported by
the product path).  ``oracle.port`` binds the C restatement gg_oracle.c;
``oracle/Makefile`` also builds the reference's own C++ into oracle/_ref/."""
