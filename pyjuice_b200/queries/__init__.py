from .sample import sample
