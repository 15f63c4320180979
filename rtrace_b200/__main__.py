import sys

from rtrace_b200.cli import main

sys.exit(main())
